"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Each fixture is the state of a small seeded box after the set-up and after given steps, produced
by the reference's C++ RT code compiled for one thread (oracle/build_ref.py; needs the reference
checkout, so this runs in the development container, not on the GPU box). The committed .npz
files pin the CPU restatement in oracle/frt_oracle.cc and, through it, the CUDA path.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

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


if __name__ == "__main__":
    for case in CASES:
        make(*case)
        print("wrote", case[0])
