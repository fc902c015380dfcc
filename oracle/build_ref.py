"""ORACLE TEST INFRASTRUCTURE -- not part of the product.

Recipe that compiles the reference's own C++/OpenMP RT code as a CPU oracle.

The reference is one translation unit built from #included .cc files (main.cc -> rt_funcs.cc ->
ray_tracing.cc -> ...), configured only through compile-time constants in user_inputs.h. It cannot
be compiled as shipped here: it #includes HEALPix 3.40 by absolute path (ray_tracing.cc:11,
mem_funcs.cc:12) and HEALPix is not installed. This recipe therefore

1. copies the reference .cc/.h files from the reference checkout into oracle/_ref/<name>/src
   (a git-ignored build directory; nothing is committed),
2. points the two HEALPix includes at oracle/healpix_shim/healpix_base.h,
3. rewrites the compile-time constants in user_inputs.h / global_variables.cc for the requested
   configuration (the reference's own configuration mechanism: go_rockfish.pbs:41-110 seds
   user_inputs.h before make),
4. compiles oracle/ref_driver.cc (which #includes the staged rt_funcs.cc chain in place of
   main.cc) with g++ -O3 -fopenmp -mcmodel=medium -ffp-contract=off.

The staged copy travels with the repository snapshot, so a box without the reference checkout can
rebuild from it (build(..., from_stage=True)) -- e.g. with a different Ncpu.
"""
from __future__ import annotations

import json
import os
import re
import shutil
import resource
import subprocess
import sys
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
# the reference checkout: FRT_REFERENCE_DIR, else the development container's checkout; a box
# without it rebuilds from the staged copies under oracle/_ref (build(..., from_stage=True))
REF_SRC = os.environ.get("FRT_REFERENCE_DIR", "/root/reference")
OUT = os.path.join(HERE, "_ref")

sys.path.insert(0, REPO)
from flexrt_imaging_reion_b200 import workloads as W  # noqa: E402

REF_FILES = ["cosmo_funcs.cc", "data_funcs.cc", "gas_funcs.cc", "general_funcs.cc", "global_constants.h",
             "global_variables.cc", "healpix_funcs.cc", "init_funcs.cc", "io_funcs.cc", "mem_funcs.cc",
             "rates.cc", "ray_tracing.cc", "rt_funcs.cc", "subgrid.cc", "user_inputs.h"]
REF_DATA = ["input_files/cosmo_table", "input_files/spectrum_tables_5bins.txt"]


def _sub_line(text: str, pattern: str, replacement: str) -> str:
    new, n = re.subn(pattern, replacement, text, count=1, flags=re.M)
    if n != 1:
        raise RuntimeError(f"pattern not found: {pattern}")
    return new


def user_inputs_values(spec: W.BoxSpec, ncpu: int, path_length: int = 8) -> dict:
    return {
        "Ncpu": ncpu, "N": spec.n, "cl_factor": spec.cl_factor(), "box": spec.box_hmpc, "zinit": spec.z,
        "ray_per_cell_max": spec.ray_per_cell_max, "path_length": path_length,
    }


def stage(name: str, spec: W.BoxSpec, ncpu: int, path_length: int = 8, restart: bool = False,
          subgrid: bool = False, ifront: bool = False) -> str:
    """Copy + configure the reference sources into oracle/_ref/<name>. A restart stage is built
    with input_grid = TRUE and reads input_files/restart_{gas,rays,tre}.bin. A sub-grid stage is
    built with subgrid = TRUE, equilibrium = TRUE, ifront = `ifront` (I-front tracking) and reads
    its tables from subgrid_files/ under the stage directory."""
    d = os.path.join(OUT, name)
    src = os.path.join(d, "src")
    os.makedirs(src, exist_ok=True)
    os.makedirs(os.path.join(d, "input_files"), exist_ok=True)
    for f in REF_FILES:
        shutil.copyfile(os.path.join(REF_SRC, f), os.path.join(src, f))
    for f in REF_DATA:
        shutil.copyfile(os.path.join(REF_SRC, f), os.path.join(d, f))
    _configure(d, spec, ncpu, path_length, restart, subgrid, ifront)
    return d


def _configure(d: str, spec: W.BoxSpec, ncpu: int, path_length: int, restart: bool = False,
               subgrid: bool = False, ifront: bool = False) -> None:
    src = os.path.join(d, "src")
    # HEALPix includes -> project shim
    for f in ("ray_tracing.cc", "mem_funcs.cc"):
        p = os.path.join(src, f)
        t = open(p).read()
        t = re.sub(r'^#include </[^>]*healpix_base\.h>', '#include "healpix_base.h"', t, flags=re.M)
        open(p, "w").write(t)
    p = os.path.join(src, "user_inputs.h")
    t = open(p).read()
    nu = ", ".join(f"{e}/h_eV" for e in W.NU_EV_5BIN)
    reps = [
        (r"^int const input_grid\s*=.*$", f"int const input_grid    = {'TRUE' if restart else 'FALSE'};"),
        (r"^const char start_file_init\[\]\s*=.*$", 'const char start_file_init[]   = "./input_files/restart_gas.bin";'),
        (r"^const char ray_file_init\[\]\s*=.*$", 'const char ray_file_init[]     = "./input_files/restart_rays.bin";'),
        (r"^const char treion_file_init\[\]\s*=.*$", 'const char treion_file_init[]  = "./input_files/restart_tre.bin";'),
        (r"^bool const c2ray_iter\s*=.*$", "bool const c2ray_iter    = TRUE;"),
        (r"^bool const ifront\s*=.*$", f"bool const ifront        = {'TRUE' if ifront else 'FALSE'};"),
        (r"^bool const he2_tr_h2\s*=.*$", "bool const he2_tr_h2     = FALSE;"),
        (r"^bool const subgrid\s*=.*$", f"bool const subgrid       = {'TRUE' if subgrid else 'FALSE'};"),
        (r"^bool const equilibrium\s*=.*$", "bool const equilibrium   = TRUE;"),
        (r"^bool const relaxed\s*=.*$", "bool const relaxed       = FALSE;"),
        (r"^const char subgrid_dir\[\]\s*=.*$", 'const char subgrid_dir[]  = "./subgrid_files/";'),
        (r"^bool const multi_freq\s*=.*$", "bool const multi_freq = TRUE;"),
        (r"^bool const MP_GADGET_HEAT\s*=.*$", "bool const MP_GADGET_HEAT = FALSE;"),
        (r"^int const Ncpu\s*=.*$", f"int const Ncpu    = {ncpu};"),
        (r"^int const Nx\s*=.*$", f"int const Nx      = {spec.n};"),
        (r"^int const Ny\s*=.*$", f"int const Ny      = {spec.n};"),
        (r"^int const Nz\s*=.*$", f"int const Nz      = {spec.n};"),
        (r"^int const Nfreq\s*=.*$", "int const Nfreq = 5;"),
        (r"^short int const hpx_lvl\s*=.*$", "short int const hpx_lvl = 0;"),
        (r"^float const tstep_factor\s*=.*$", "float const tstep_factor = 1.0;"),
        (r"^float const cl_factor\s*=.*$", f"float const cl_factor    = {spec.cl_factor()!r};"),
        (r"^int const itercount\s*=.*$", "int const itercount      = 5;"),
        (r"^float const safety_factor\s*=.*$", "float const safety_factor = 3.;"),
        (r"^float const const_clump\s*=.*$", "float const const_clump = 1.0;"),
        (r"^float const zinit\s*=.*$", f"float const zinit    = {spec.z!r};"),
        (r"^float const fesc\s*=.*$", "float const fesc                = 1.0;"),
        (r"^float const Lx0\s*=.*$", f"float const Lx0 = {spec.box_hmpc!r}*1e3/hh;"),
        (r"^float const Ly0\s*=.*$", f"float const Ly0 = {spec.box_hmpc!r}*1e3/hh;"),
        (r"^float const Lz0\s*=.*$", f"float const Lz0 = {spec.box_hmpc!r}*1e3/hh;"),
        (r"^double const nu_phot\[Nfreq\]\s*=.*$", f"double const nu_phot[Nfreq] = {{{nu}}};"),
        (r"^float const temp_0\s*=.*$", "float const temp_0 = 1e4;"),
        (r"^int const path_length\s*=.*$", f"int const path_length = {path_length};"),
        # file names of update_hydro_step (gas_funcs.cc:554-752), relative to the stage directory
        # (ref_driver's FRT_HYDRO hook)
        (r"^const int snapinit\s*=.*$", "const int snapinit             = 10;"),
        (r"^const char output_dir\[\]\s*=.*$", 'const char output_dir[]      = "./hydro_out/";'),
        (r"^const char hydro_base\[\]\s*=.*$", 'const char hydro_base[]    = "./hydro/";'),
        (r"^const char density_dir\[\]\s*=.*$", 'const char density_dir[] = "";'),
        (r"^const char source_dir\[\]\s*=.*$", 'const char source_dir[] = "";'),
    ]
    for pat, rep in reps:
        t = _sub_line(t, pat, rep)
    open(p, "w").write(t)
    p = os.path.join(src, "global_variables.cc")
    t = open(p).read()
    t = _sub_line(t, r"^short int const ray_per_cell_max\s*=.*$",
                  f"short int const ray_per_cell_max = {spec.ray_per_cell_max};")
    open(p, "w").write(t)
    json.dump({"name": os.path.basename(d), "ncpu": ncpu, "path_length": path_length, "subgrid": subgrid,
               "ifront": ifront,
               "spec": __import__("dataclasses").asdict(spec)},
              open(os.path.join(d, "stage.json"), "w"), indent=1)


def compile_stage(d: str, ncpu: Optional[int] = None) -> str:
    """Compile ref_driver against the staged sources; optionally re-set Ncpu first."""
    src = os.path.join(d, "src")
    if ncpu is not None:
        p = os.path.join(src, "user_inputs.h")
        t = open(p).read()
        t = _sub_line(t, r"^int const Ncpu\s*=.*$", f"int const Ncpu    = {ncpu};")
        open(p, "w").write(t)
        meta = json.load(open(os.path.join(d, "stage.json")))
        meta["ncpu"] = ncpu
        json.dump(meta, open(os.path.join(d, "stage.json"), "w"), indent=1)
    exe = os.path.join(d, "ref_driver")
    cmd = ["g++", "-O3", "-fopenmp", "-mcmodel=medium", "-ffp-contract=off", "-w", "-std=gnu++17",
           "-I", src, "-I", os.path.join(HERE, "healpix_shim"), "-I", HERE,
           os.path.join(HERE, "ref_driver.cc"), "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def build(name: str, spec: W.BoxSpec, ncpu: int = 1, path_length: int = 8, from_stage: bool = False,
          restart: bool = False, subgrid: bool = False, ifront: bool = False) -> str:
    d = os.path.join(OUT, name)
    if not from_stage:
        if not os.path.isdir(REF_SRC):
            raise RuntimeError("reference checkout not available; use from_stage=True")
        stage(name, spec, ncpu, path_length, restart, subgrid, ifront)
        return compile_stage(d)
    return compile_stage(d, ncpu)


def _unlimited_stack():
    # update_thermal keeps a float[Nx][Ny][Nz] array on the stack (gas_funcs.cc:364)
    try:
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        soft, hard = resource.getrlimit(resource.RLIMIT_STACK)
        resource.setrlimit(resource.RLIMIT_STACK, (hard, hard))


def run(name: str, inp: W.BoxInputs, rundir: str, nsteps: int, seed: int, dump_every: int = 1,
        threads: int = 1, timeout: Optional[float] = None, restart_out: Optional[str] = None,
        cosmo: bool = False, hydro=None) -> str:
    """Run the compiled reference on inputs written to rundir; returns stdout. With restart_out,
    the reference's restart writers store gas.bin / rays.bin / tre.bin there after the last step;
    with cosmo, the cosmological expansion runs after every step (its scale factors are logged as
    'COSMO step a_current a_prev' lines)."""
    d = os.path.join(OUT, name)
    W.write_reference_inputs(inp, rundir)
    args = [os.path.join(d, "ref_driver"), os.path.abspath(rundir), str(nsteps), str(seed), str(dump_every),
            repr(inp.spec.rkill_cm())]
    if inp.clump is not None:
        args.append(os.path.join(os.path.abspath(rundir), "clump.bin"))
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    if restart_out:
        env["FRT_RESTART_OUT"] = os.path.abspath(restart_out)
    if cosmo:
        env["FRT_COSMO"] = "1"
    if hydro:
        # snapshot switches: ([step, ...], [z1, z2, z3], [BoxInputs of snapshot 1, 2])
        at, zs, snaps = hydro
        os.makedirs(os.path.join(d, "hydro"), exist_ok=True)
        os.makedirs(os.path.join(d, "hydro_out"), exist_ok=True)
        for n, snap in enumerate(snaps, 1):
            tag = f"01{n}"
            snap.delta1.astype("float32").tofile(os.path.join(d, "hydro", f"density.{tag}.{snap.spec.n}"))
            cat = np.zeros((snap.src_pos.shape[0], 5), dtype=np.float64)
            cat[:, 0:3] = snap.src_pos
            cat[:, 4] = snap.src_lum
            cat.tofile(os.path.join(d, "hydro", f"ndot_catalog_{tag}"))
            np.array([snap.src_pos.shape[0]], dtype=np.int64).tofile(os.path.join(d, "hydro", f"numhalos.{tag}"))
        env["FRT_HYDRO"] = ",".join(str(k) for k in at)
        env["FRT_HYDRO_Z"] = ",".join(repr(float(z)) for z in zs)
    r = subprocess.run(args, cwd=d, env=env, capture_output=True, text=True, timeout=timeout,
                       preexec_fn=_unlimited_stack)
    if r.returncode != 0:
        raise RuntimeError(f"ref_driver failed ({r.returncode}): {r.stdout[-2000:]} {r.stderr[-2000:]}")
    return r.stdout


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("config")
    ap.add_argument("--name")
    ap.add_argument("--ncpu", type=int, default=1)
    a = ap.parse_args()
    spec = W.CONFIGS[a.config]() if a.config in W.CONFIGS else W.config_tiny()
    print(build(a.name or a.config, spec, a.ncpu))
