"""Several independent boxes of different sizes in one context (the uneven-ensemble form): each
box must match the oracle run of that box alone, with the contract tolerances of
tests/test_gpu_parity.py, in the fused graph step and in the plain per-kernel launch form."""
import numpy as np
import pytest

import parity_tools as PT
from flexrt_imaging_reion_b200 import rt, workloads as W
from test_gpu_parity import check

pytestmark = pytest.mark.gpu

BOXES = [
    (W.config_tiny(n=16, n_src=5, steps=6, seed=31, name="B16"), 101),
    # a box that reaches the merge threshold in the last step
    (W.config_tiny(n=20, n_src=10, steps=6, seed=32, name="B20", ray_per_cell_max=13, lum_min=1e53, lum_max=1e55), 102),
    (W.config_tiny(n=32, n_src=3, steps=6, seed=33, name="B32", sigma_ln=0.8, z=7.0), 103),
]


@pytest.fixture(scope="module")
def oracle_runs():
    return [PT.oracle_states(W.make_inputs(spec), seed, spec.steps) for spec, seed in BOXES]


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("precision", ["strict", "mixed"])
def test_ensemble_matches_per_box_oracle(oracle_runs, graph, precision):
    inputs = [W.make_inputs(spec) for spec, _ in BOXES]
    ctx = rt.RTContext(inputs, [seed for _, seed in BOXES], precision=precision, outputs="diag",
                       ray_capacity=1 << 20)
    ctx.setup()
    steps = BOXES[0][0].steps
    states = [[PT.device_state(ctx, b, True)] for b in range(len(BOXES))]
    for _ in range(steps):
        st = ctx.step(graph=graph)
        for b in range(len(BOXES)):
            states[b].append(PT.device_state(ctx, b, True))
        # crossings summed over the boxes
        s = len(states[0]) - 1
        assert st["crossings"] == sum(int(r[s]["scalars"][10]) for r in oracle_runs)
    for b in range(len(BOXES)):
        check(states[b], oracle_runs[b], precision == "strict", merged=True)
        # each box kept its own time step (dt follows the box's cell size and redshift)
        dt_dev = ctx.box_scalars(b)["dt"]
        assert abs(dt_dev - float(oracle_runs[b][-1]["scalars"][1])) <= 1e-6 * dt_dev
    assert float(oracle_runs[1][-1]["scalars"][4]) > 0   # merging happened in box B20
    ctx.close()


def test_ensemble_photon_budget():
    inputs = [W.make_inputs(spec) for spec, _ in BOXES]
    ctx = rt.RTContext(inputs, [seed for _, seed in BOXES], precision="mixed", ray_capacity=1 << 20)
    ctx.setup()
    in0 = ctx.in_flight()
    stats = [ctx.step() for _ in range(4)]
    assert PT.photon_budget(stats, in0) < 1e-6
    ctx.close()
