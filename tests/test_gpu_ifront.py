"""I-front tracking on the device (frt_set_subgrid with ifront) against the oracle, whose
restatement is pinned bit for bit on the reference's own code with ifront = TRUE
(tests/test_ifront_oracle.py, tests/golden/T16F.npz): T16 over 8 steps in which the fronts cross
many cells part-way, every step at the contract tolerances of tests/test_gpu_parity.py, and the
front state of every cell: the passed fraction, its maximum, the crossing times (total and per
tenth of the cell) and the flags.

The neutral part of a cell absorbs the rays' photons in the order of the reference's slots, so
the device keeps its rays in that order and resolves the budgets by rounds to a fixed point; the
ray multiset, the ionised flags and the front fractions follow the oracle's sequential walk."""
import os
import sys
import tempfile

import numpy as np
import pytest

import parity_tools as PT
from flexrt_imaging_reion_b200 import rt, workloads as W
from oracle import frtd, oracle as O
from test_gpu_parity import check

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import subgrid_tables as ST  # noqa: E402

pytestmark = pytest.mark.gpu

G = np.load(os.path.join(HERE, "golden", "T16F.npz"))
SPEC = W.config_tiny(steps=8)
TABLES = ST.reference_arrays(*G["span"])
FRONT = {"fion": "FION", "fion_max": "FION_MAX", "tcross": "TCROSS", "tcross_new": "TCROSS_NEW",
         "tcross_flag": "TCROSS_FLAG", "neutral_flag": "NEUTRAL_FLAG"}


def oracle_states(spec=SPEC, seed=int(G["seed"]), steps=SPEC.steps):
    o = O.Oracle(W.make_inputs(spec), seed)
    o.set_subgrid(TABLES, G["consts"], ifront=True)
    out = []
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "x.frtd")
        for s in range(steps + 1):
            if s > 0:
                o.step()
            o.dump(p)
            out.append(frtd.read(p))
    o.close()
    return out


def device_run(precision, outputs, mode, spec=SPEC, seed=int(G["seed"]), steps=SPEC.steps):
    ctx = rt.RTContext([W.make_inputs(spec)], [seed], precision=precision, outputs=outputs,
                       ray_capacity=1 << 20)
    ctx.setup()
    ctx.set_subgrid(TABLES, G["consts"], ifront=True)
    diag = outputs == "diag"

    def snap():
        st = PT.device_state(ctx, 0, diag)
        for k, f in FRONT.items():
            st[k] = ctx.get_field(0, f)
        st["mfp"] = ctx.get_field(0, "MFP")
        return st

    states, stats = [snap()], []
    for _ in range(steps):
        if mode == "unfused":
            ctx.step_unfused()
            stats.append(ctx.last_stats())
        else:
            stats.append(ctx.step(graph=(mode == "graph")))
        states.append(snap())
    ctx.close()
    return states, stats


@pytest.mark.parametrize("precision,outputs,mode", [("strict", "diag", "graph"), ("mixed", "core", "graph"),
                                                    ("strict", "diag", "unfused")])
def test_ifront_matches_oracle(precision, outputs, mode):
    ref = oracle_states()
    states, stats = device_run(precision, outputs, mode)
    check(states, ref, True, stats=None if mode == "unfused" else stats)
    for s in range(1, len(states)):
        d, r = states[s], ref[s]
        for k in ("tcross_flag", "neutral_flag"):
            np.testing.assert_array_equal(d[k] != 0, r[k] != 0, err_msg=f"step {s} {k}")
        for k in ("fion", "fion_max"):
            np.testing.assert_allclose(d[k], r[k], rtol=1e-5, atol=1e-6, err_msg=f"step {s} {k}")
        dt = float(r["scalars"][1])
        for k in ("tcross", "tcross_new"):   # times: to 1e-5 of the time step
            np.testing.assert_allclose(d[k], r[k], rtol=1e-6, atol=1e-5 * dt, err_msg=f"step {s} {k}")
        if mode != "unfused":
            assert stats[s - 1]["crossings"] == int(r["scalars"][10]), s
    # the fronts were tracked: cells part-way ionised and rays absorbed whole in neutral cells
    f = ref[-1]["fion"]
    assert int(((f > 0) & (f < 1)).sum()) > 100


def test_ifront_s_box():
    """The S box (64^3, 32 sources) with I-front tracking over 4 steps, on the T16F tables and
    cosmic times: many more rays share each front cell, so the budgets take more rounds."""
    spec, seed, steps = W.config_S(), 21, 4
    ref = oracle_states(spec, seed, steps)
    states, stats = device_run("mixed", "core", "graph", spec, seed, steps)
    check(states, ref, False, stats=stats)
    for s in range(1, len(states)):
        d, r = states[s], ref[s]
        np.testing.assert_array_equal(d["tcross_flag"] != 0, r["tcross_flag"] != 0, err_msg=f"step {s}")
        np.testing.assert_allclose(d["fion"], r["fion"], rtol=1e-4, atol=1e-5, err_msg=f"step {s} fion")
        assert stats[s - 1]["crossings"] == int(r["scalars"][10]), s
    assert int(((ref[-1]["fion"] > 0) & (ref[-1]["fion"] < 1)).sum()) > 100
