"""The opt-in optical-depth limit on the device against the oracle's restatement of the same rule.

frt_set_tau_limit(5): each ray carries its HI and HeI columns in FP64 and is removed once its
optical depth exceeds 5 in every bin (a rule of the hot-path specification that the reference does
not have, so parity is pinned on the oracle only). The 16^3 box over 8 steps in both precisions:
the contract tolerances of tests/test_gpu_parity.py on every field, the ray tree and the photon
ledger, each matched ray's columns (sums of the cells' time-averaged densities, which the device
forms from float-atomic rate sums: 1e-4 relative in mixed precision, 1e-5 in strict, the rates'
tolerances), and a ray kept on one side only must tie with nphot_min or with the limit. The limit must remove rays the reference rule keeps.
"""
import numpy as np
import pytest

import parity_tools as PT
from flexrt_imaging_reion_b200 import rt, workloads as W
from test_gpu_parity import check

pytestmark = pytest.mark.gpu

SPEC, SEED, TAU = W.config_tiny(n=16, n_src=6, steps=8), 11, 5.0


def _device(precision, tau):
    ctx = rt.RTContext([W.make_inputs(SPEC)], [SEED], precision=precision, outputs="diag", ray_capacity=1 << 20)
    ctx.setup()
    if tau > 0:
        ctx.set_tau_limit(tau)
    states, stats = [], []

    def grab():
        st = PT.device_state(ctx, 0, True)
        st["ray_col"] = ctx.ray_columns(0)
        states.append(st)

    grab()
    for _ in range(SPEC.steps):
        stats.append(ctx.step(graph=True))
        grab()
    ctx.close()
    return states, stats


@pytest.mark.parametrize("precision", ["strict", "mixed"])
def test_tau_limit_matches_oracle(precision):
    ref = PT.oracle_states(W.make_inputs(SPEC), SEED, SPEC.steps, tau_max=TAU)
    states, stats = _device(precision, TAU)
    strict = precision == "strict"
    check(states, ref, strict, stats=stats)
    for s in range(1, SPEC.steps + 1):
        r = PT.compare_rays(states[s], ref[s], ref[s]["scalars"][2], 1e-5 if strict else 1e-4,
                            dx=float(ref[s]["scalars"][8]), dx0=float(ref[s]["scalars"][7]))
        assert r["col_maxrel"] < (1e-5 if strict else 1e-4), (s, r["col_maxrel"])
    # the limit removed rays that the nphot_min rule alone keeps
    off, _ = _device(precision, 0.0)
    assert len(states[-1]["ray_order"]) < len(off[-1]["ray_order"])
    assert np.count_nonzero(states[-1]["ray_col"][:, 0]) > 0
