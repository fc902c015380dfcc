"""The sub-grid model on the device (frt_set_subgrid) against the oracle, whose restatement is
pinned bit for bit on the reference's own sub-grid code (tests/test_subgrid_oracle.py,
tests/golden/T16G.npz): T16 over 6 steps in which the ionised region grows, on the synthetic
RadHydro and overdensity tables, every step at the contract tolerances of
tests/test_gpu_parity.py (ledger included), and the equilibrium mean free path of every cell."""
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

G = np.load(os.path.join(HERE, "golden", "T16G.npz"))
SPEC = W.config_tiny(steps=6)
TABLES = ST.reference_arrays(*G["span"])


def oracle_states():
    o = O.Oracle(W.make_inputs(SPEC), int(G["seed"]))
    o.set_subgrid(TABLES, G["consts"])
    out = []
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "x.frtd")
        for s in range(SPEC.steps + 1):
            if s > 0:
                o.step()
            o.dump(p)
            out.append(frtd.read(p))
    o.close()
    return out


def device_run(precision, outputs, mode):
    ctx = rt.RTContext([W.make_inputs(SPEC)], [int(G["seed"])], precision=precision, outputs=outputs,
                       ray_capacity=1 << 20)
    ctx.setup()
    ctx.set_subgrid(TABLES, G["consts"])
    diag = outputs == "diag"
    states, stats, mfp = [PT.device_state(ctx, 0, diag)], [], [ctx.get_field(0, "MFP")]
    for _ in range(SPEC.steps):
        if mode == "unfused":
            ctx.step_unfused()
            stats.append(ctx.last_stats())
        else:
            stats.append(ctx.step(graph=(mode == "graph")))
        states.append(PT.device_state(ctx, 0, diag))
        mfp.append(ctx.get_field(0, "MFP"))
    ctx.close()
    return states, stats, mfp


@pytest.mark.parametrize("precision,outputs,mode", [("strict", "diag", "graph"), ("strict", "diag", "unfused"),
                                                    ("mixed", "core", "graph"), ("mixed", "diag", "plain")])
def test_subgrid_matches_oracle(precision, outputs, mode):
    ref = oracle_states()
    states, stats, mfp = device_run(precision, outputs, mode)
    check(states, ref, True, stats=None if mode == "unfused" else stats)
    for s in range(len(states)):
        # the equilibrium mean free path: one rounding of the reference's own expression
        lit = ref[s]["treion_flag"] != 0
        r = PT._rel(mfp[s], ref[s]["mfp"], 1e-30)
        assert float(r[lit].max(initial=0.0)) < 1e-5, (s, float(r[lit].max(initial=0.0)))
        assert float(r[~lit].max(initial=0.0)) < 1e-6, s
        if mode != "unfused" and s > 0:
            assert stats[s - 1]["crossings"] == int(ref[s]["scalars"][10]), s
    # the model ran: cells ionised and HI fractions from the tables, below the plain model's
    assert int(ref[-1]["treion_flag"].sum()) > 100
    np.testing.assert_array_equal(states[-1]["treion_flag"], ref[-1]["treion_flag"])


def test_subgrid_refusals():
    """The phased step, the autotuner and the adjoint stay with the plain model."""
    ctx = rt.RTContext([W.make_inputs(SPEC)], [int(G["seed"])], precision="mixed", outputs="core",
                       ray_capacity=1 << 20)
    ctx.setup()
    ctx.set_subgrid(TABLES, G["consts"])
    with pytest.raises(rt.FrtError):
        ctx.autotune(1)
    ctx.step()
    with pytest.raises(rt.FrtError):
        ctx.adjoint((0, 0, 0), (4, 4, 4))
    ctx.close()
