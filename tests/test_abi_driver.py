"""The C ABI from a compiled C++ caller (tests/abi_driver.cc), not only through the ctypes mirror.

The driver includes include/flexrt.h, links libflexrt_b200.so and replays the reference driver's
set-up and step loop (main.cc:10-264) through the entry points. On the CPU: it compiles against the
header, and the struct layouts the compiler gives it are the ones the ctypes mirror
(flexrt_imaging_reion_b200/_abi.py) declares. On the GPU: two steps of the S box, through the
individual step functions and through frt_step, with the oracle's crossings per step.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import parity_tools as PT
from flexrt_imaging_reion_b200 import _abi, rt, workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def driver(product_lib, tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("abi") / "abi_driver")
    libdir = os.path.dirname(_abi.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"),
                    os.path.join(HERE, "abi_driver.cc"), "-L", libdir, "-lflexrt_b200", f"-Wl,-rpath,{libdir}",
                    "-o", exe], check=True)
    return exe


def _offsets(struct):
    return {name: getattr(struct, name).offset for name, _ in struct._fields_}


def test_struct_layouts_match_compiled_header(driver):
    out = subprocess.run([driver, "layout"], check=True, capture_output=True, text=True).stdout
    rows = {}
    for line in out.splitlines():
        tok = line.split()
        rows[tok[0]] = (int(tok[1]), {tok[k]: int(tok[k + 1]) for k in range(2, len(tok), 2)})
    for cname, struct in (("frt_box_desc", _abi.BoxDesc), ("frt_config", _abi.Config),
                          ("frt_step_stats", _abi.StepStats), ("frt_adj_objective", _abi.AdjObjective)):
        size, offs = rows[cname]
        assert size == C.sizeof(struct), cname
        assert offs == _offsets(struct), cname


def _write_box(d, spec, seed):
    inp = W.make_inputs(spec)
    ijk, lum = W.grid_sources(inp)
    with open(os.path.join(d, "box.txt"), "w") as f:
        f.write(f"{spec.n} {spec.box_hmpc!r} {spec.z!r} {spec.cl_factor()!r} {spec.rkill_cm()!r} {seed} {len(lum)}\n")
    spec_f = rt.spectrum_alpha15()
    with open(os.path.join(d, "spectrum.txt"), "w") as f:
        f.write(f"{len(spec_f)}\n")
        for e, fr in zip(W.NU_EV_5BIN, spec_f):
            f.write(f"{e / W.H_EV!r} {float(fr)!r}\n")
    np.ascontiguousarray(inp.delta1, np.float32).tofile(os.path.join(d, "density.bin"))
    np.ascontiguousarray(ijk, np.int32).tofile(os.path.join(d, "src_ijk.bin"))
    np.ascontiguousarray(lum, np.float64).tofile(os.path.join(d, "src_lum.bin"))
    return inp


@pytest.mark.gpu
@pytest.mark.parametrize("fused", [0, 1])
def test_driver_steps_s_box(driver, tmp_path, fused):
    spec, seed, steps = W.config_S(), 21, 2
    inp = _write_box(str(tmp_path), spec, seed)
    r = subprocess.run([driver, "run", str(tmp_path), str(steps), str(fused)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l.split() for l in r.stdout.splitlines() if l.startswith("STEP")]
    assert len(lines) == steps, r.stdout
    ref = PT.oracle_states(inp, seed, steps)
    for s, tok in enumerate(lines, 1):
        assert int(tok[2]) == 0, tok                                # status
        assert int(tok[3]) == int(ref[s]["scalars"][10]), (s, tok)   # crossings of the step
        assert int(tok[4]) == len(ref[s]["ray_order"]), (s, tok)     # live rays after the step
