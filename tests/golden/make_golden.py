"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Each fixture is the state of a small seeded box after the set-up and after given steps, produced
by the reference's C++ RT code compiled for one thread (oracle/build_ref.py; needs the reference
checkout, so this runs in the development container, not on the GPU box). The committed .npz
files pin the CPU restatement in oracle/frt_oracle.cc and, through it, the CUDA path.

    python tests/golden/make_golden.py [names]

T16C holds a run with the reference's cosmological expansion after every step and the scale
factors it used. T16G and T16F run the sub-grid model on synthetic RadHydro tables, without and with
I-front tracking. T16H adds two hydro snapshot switches (update_hydro_step) with rays in flight. T16R holds the reference's restart files (write_gas_binary / write_rays_binary / write_treion
after 3 steps of T16) and the states of the reference's own restart path run from them.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from oracle import build_ref as B, frtd  # noqa: E402
from flexrt_imaging_reion_b200 import workloads as W  # noqa: E402

FIELDS = ["nH1", "nHe1", "f_H1", "f_He1", "temp", "avg_nh1", "avg_nhe1", "gamma_H1_tot", "gamma_He1_tot",
          "heat_rate", "cool_rate", "ne", "treion", "treion_flag", "gamma_H1_nu", "ngam_nu", "mfp", "recrate_H2"]
RAYS = ["ray_active", "ray_order", "ray_pixel", "ray_itheta", "ray_cell", "ray_end", "ray_geom", "ray_nphot"]

# (name, spec, seed, steps to keep)
CASES = [
    ("T16", W.config_tiny(), 11, [1, 6]),
    ("T16M", W.config_tiny(n=16, n_src=6, steps=6, seed=5, name="T16M", clump_model="sqrt", ray_per_cell_max=12),
     3, [6]),
    ("T16N", W.config_tiny(n=16, n_src=10, steps=8, seed=9, name="T16N", ray_per_cell_max=13, lum_min=1e53,
                           lum_max=1e55), 4, [8]),
]


def make(name, spec, seed, keep):
    B.build(name, spec, ncpu=1)
    inp = W.make_inputs(spec)
    out = {}
    with tempfile.TemporaryDirectory() as td:
        B.run(name, inp, td, spec.steps, seed, dump_every=1)
        for s in keep:
            d = frtd.read(os.path.join(td, f"dump_{s:04d}.frtd"))
            for k in FIELDS:
                out[f"s{s}_{k}"] = d[k]
            for k in RAYS:
                out[f"s{s}_{k}"] = d[k]
            out[f"s{s}_scalars"] = d["scalars"]
            out[f"s{s}_spectrum"] = d["spectrum"]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), seed=seed, steps=np.array(keep), **out)


def compact_ray_slots(raw: bytes, nfreq: int = 5) -> bytes:
    """The same ray records with slot numbers 0..n-1 (the reference's reader takes any slot; with
    no holes, rays cast after the restart take the slots after the loaded ones, so the slot order
    stays the creation order the oracle keeps)."""
    rec = 8 + 1 + 2 + 4 + 2 + 12 + 4 * nfreq + 24 + 4
    out = bytearray()
    pos, x = 0, 0
    while True:
        slot = int(np.frombuffer(raw[pos:pos + 8], np.int64)[0])
        if slot == -1:
            break
        out += np.int64(x).tobytes() + raw[pos + 8:pos + rec]
        pos += rec
        x += 1
    out += np.int64(-1).tobytes()
    return bytes(out)


def make_restart(name="T16R", base=("T16", W.config_tiny(), 11), steps_before=3, steps_after=2, seed=21):
    """The reference's restart files after `steps_before` steps of a fresh run (its own writers),
    and the states of a run of the reference's restart path (input_grid = TRUE) from them."""
    bname, spec, bseed = base
    B.build(bname, spec, ncpu=1)
    B.build(name, spec, ncpu=1, restart=True)
    inp = W.make_inputs(spec)
    out = {}
    with tempfile.TemporaryDirectory() as td:
        rs = os.path.join(td, "rs")
        os.makedirs(rs)
        B.run(bname, inp, os.path.join(td, "a"), steps_before, bseed, dump_every=0, restart_out=rs)
        raw = {k: open(os.path.join(rs, f"{k}.bin"), "rb").read() for k in ("gas", "rays", "tre")}
        comp = compact_ray_slots(raw["rays"])
        d = os.path.join(B.OUT, name, "input_files")
        for k, v in (("gas", raw["gas"]), ("rays", comp), ("tre", raw["tre"])):
            open(os.path.join(d, f"restart_{k}.bin"), "wb").write(v)
        B.run(name, inp, os.path.join(td, "b"), steps_after, seed, dump_every=1)
        for s in range(1, steps_after + 1):
            dd = frtd.read(os.path.join(td, "b", f"dump_{s:04d}.frtd"))
            for k in FIELDS + RAYS + ["scalars"]:
                out[f"s{s}_{k}"] = dd[k]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), seed=seed, base_seed=bseed, steps_before=steps_before,
                        steps=np.arange(1, steps_after + 1),
                        gas=np.frombuffer(raw["gas"], np.uint8), rays=np.frombuffer(raw["rays"], np.uint8),
                        rays_compact=np.frombuffer(comp, np.uint8), tre=np.frombuffer(raw["tre"], np.uint8), **out)


def make_cosmo(name="T16C", base=("T16", W.config_tiny(), 11), steps=4):
    """A fresh run with the cosmological expansion after every step (the reference's own
    update_cosmo_expansion), its states and the scale factors each expansion used."""
    bname, spec, seed = base
    B.build(bname, spec, ncpu=1)
    inp = W.make_inputs(spec)
    out = {}
    with tempfile.TemporaryDirectory() as td:
        log = B.run(bname, inp, td, steps, seed, dump_every=1, cosmo=True)
        ac, ap = [], []
        for line in log.splitlines():
            if line.startswith("COSMO"):
                _, s, a, b = line.split()
                ac.append(float.fromhex(a))
                ap.append(float.fromhex(b))
        assert len(ac) == steps
        for s in range(1, steps + 1):
            dd = frtd.read(os.path.join(td, f"dump_{s:04d}.frtd"))
            for k in FIELDS + RAYS + ["scalars"]:
                out[f"s{s}_{k}"] = dd[k]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), seed=seed, steps=np.arange(1, steps + 1),
                        a_current=np.array(ac, np.float32), a_prev=np.array(ap, np.float32), **out)


HYDRO_Z = (7.9, 7.8, 7.7)   # the redshifts of snapshots 1, 2 and the one after them
HYDRO_AT = (2, 4)           # switches after these steps


def hydro_snapshots(spec):
    """The later snapshots of the snapshot-switch case: the same box, its own seeded density and
    sources per snapshot (seeds 101, 102)."""
    import dataclasses
    return [W.make_inputs(dataclasses.replace(spec, seed=100 + n, sigma_ln=0.5 + 0.05 * n)) for n in (1, 2)]


def make_hydro(name="T16H", base=("T16", W.config_tiny(), 11), steps=6):
    """A run with the cosmological expansion after every step and two hydro snapshot switches
    (the reference's own update_hydro_step and get_nphot_min_max) after steps 2 and 4, with rays
    in flight: its states, the scale factors of every expansion and the (a_rt, dt_snap, zz) of
    every switch. The second switch is the first with a previous snapshot, so d(delta)/dt enters
    the temperature equation from then on."""
    bname, spec, seed = base
    B.build(bname, spec, ncpu=1)
    inp = W.make_inputs(spec)
    snaps = hydro_snapshots(spec)
    out = {}
    with tempfile.TemporaryDirectory() as td:
        log = B.run(bname, inp, td, steps, seed, dump_every=1, cosmo=True, hydro=(HYDRO_AT, HYDRO_Z, snaps))
        ac, ap, hy = [], [], []
        for line in log.splitlines():
            if line.startswith("COSMO"):
                _, s_, a, b = line.split()
                ac.append(float.fromhex(a))
                ap.append(float.fromhex(b))
            if line.startswith("HYDRO"):
                _, s_, a, dts, z = line.split()
                hy.append([float(int(s_)), float.fromhex(a), float.fromhex(dts), float.fromhex(z)])
        assert len(ac) == steps and len(hy) == len(HYDRO_AT), log[-2000:]
        for s in range(1, steps + 1):
            dd = frtd.read(os.path.join(td, f"dump_{s:04d}.frtd"))
            for k in FIELDS + RAYS + ["scalars"]:
                out[f"s{s}_{k}"] = dd[k]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), seed=seed, steps=np.arange(1, steps + 1),
                        a_current=np.array(ac, np.float32), a_prev=np.array(ap, np.float32),
                        hydro=np.array(hy, np.float64), **out)


IFRONT_FIELDS = ["fion", "fion_max", "tcross", "tcross_new", "tcross_flag", "neutral_flag", "Delta_fion", "IF_speed",
                 "Inc_Flux", "treion_out"]


def make_subgrid(name="T16G", base=("T16", W.config_tiny(steps=6), 11), steps=6, ifront=False):
    """A run of the reference's sub-grid model (subgrid = TRUE, equilibrium = TRUE, ifront as
    given) on synthetic tables in its own file formats (tests/golden/subgrid_tables.py): its
    states, the cosmic times the model used (logged by the reference) and the span of the
    overdensity table, so that the tables can be rebuilt without the reference's cosmology
    table. With I-front tracking the states also hold the front fractions and crossing times."""
    import subgrid_tables as ST
    _, spec, seed = base
    B.build(name, spec, ncpu=1, subgrid=True, ifront=ifront)
    d = os.path.join(B.OUT, name)
    ct = ST.cosmic_time_from_table(os.path.join(d, "input_files", "cosmo_table"))
    t0, t1 = ST.table_span(ct)
    ST.write_reference_files(os.path.join(d, "subgrid_files"), ct)
    inp = W.make_inputs(spec)
    out = {}
    with tempfile.TemporaryDirectory() as td:
        log = B.run(name, inp, td, steps, seed, dump_every=1)
        consts = None
        for line in log.splitlines():
            if line.startswith("SUBGRID"):
                consts = [float.fromhex(x) for x in line.split()[1:]]
        assert consts is not None and len(consts) == 7, log[-2000:]
        for s in range(1, steps + 1):
            dd = frtd.read(os.path.join(td, f"dump_{s:04d}.frtd"))
            for k in FIELDS + RAYS + ["scalars", "mfp", "f_H2"] + (IFRONT_FIELDS if ifront else []):
                out[f"s{s}_{k}"] = dd[k]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), seed=seed, steps=np.arange(1, steps + 1),
                        consts=np.array(consts, np.float32), span=np.array([t0, t1], np.float64), **out)


if __name__ == "__main__":
    only = sys.argv[1:]
    for case in CASES:
        if not only or case[0] in only:
            make(*case)
            print("wrote", case[0])
    if not only or "T16R" in only:
        make_restart()
        print("wrote T16R")
    if not only or "T16C" in only:
        make_cosmo()
        print("wrote T16C")
    if not only or "T16H" in only:
        make_hydro()
        print("wrote T16H")
    if not only or "T16G" in only:
        make_subgrid()
        print("wrote T16G")
    if not only or "T16F" in only:
        make_subgrid(name="T16F", steps=8, ifront=True)
        print("wrote T16F")
