"""The cosmological expansion between steps on the device (frt_update_cosmo_expansion) against
the oracle's (pinned bit for bit on the reference's update_cosmo_expansion by
tests/test_cosmo_oracle.py), fed the scale factors of tests/golden/T16C.npz, with the parity
tolerances of tests/test_gpu_parity.py after every step."""
import os
import tempfile

import numpy as np
import pytest

import parity_tools as PT
from flexrt_imaging_reion_b200 import rt, workloads as W
from oracle import frtd, oracle as O
from test_gpu_parity import check

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "T16C.npz"))
SPEC = W.config_tiny()


def _oracle_states(inp, seed):
    o = O.Oracle(inp, seed)
    out = []
    with tempfile.TemporaryDirectory() as td:
        for s in G["steps"]:
            o.step()
            o.cosmo_expansion(float(G["a_current"][s - 1]), float(G["a_prev"][s - 1]))
            p = os.path.join(td, "x.frtd")
            o.dump(p)
            out.append(frtd.read(p))
    o.close()
    return out


@pytest.mark.parametrize("precision,graph", [("strict", True), ("mixed", True), ("mixed", False)])
def test_expansion_matches_oracle(precision, graph):
    inp = W.make_inputs(SPEC)
    seed = int(G["seed"])
    ref = _oracle_states(inp, seed)
    ctx = rt.RTContext([inp], [seed], precision=precision, outputs="diag", ray_capacity=1 << 20)
    ctx.setup()
    states = []
    for s in G["steps"]:
        ctx.step(graph=graph)
        ctx.cosmo_expansion(G["a_current"][s - 1], G["a_prev"][s - 1])
        states.append(PT.device_state(ctx, 0, True))
        sc = ctx.box_scalars(0)
        # cell size and time step follow the expansion exactly (update_dt, float arithmetic)
        assert np.float32(sc["dx"]) == np.float32(ref[s - 1]["scalars"][8])
        assert np.float32(sc["dt"]) == np.float32(ref[s - 1]["scalars"][1])
    rho = ctx.get_field(0, "RHO")
    ctx.close()
    check(states, ref, precision == "strict", merged=True)
    np.testing.assert_array_equal(rho, ref[-1]["rho"])
