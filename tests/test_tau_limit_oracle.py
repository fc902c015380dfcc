"""The opt-in optical-depth limit in the oracle (no counterpart in the reference, whose rays end
only below nphot_min, ray_tracing.cc:782, 927-933).

With tau_max > 0 every ray carries the HI and HeI columns it crossed since its cast, summed in FP64
over the segments of each step's last C2Ray iteration, and a ray whose optical depth exceeds
tau_max in every bin is removed after the step's last ray pass. Parity against the reference is
unpinned by construction (the rule is not the reference's); these checks pin the restatement's
own properties, and tests/test_gpu_tau_limit.py holds the device to it.
"""
import numpy as np

import parity_tools as PT
from flexrt_imaging_reion_b200 import workloads as W

SPEC, SEED, TAU = W.config_tiny(n=16, n_src=6, steps=8), 11, 5.0


def _tau_min(st):
    sig = st["tau_sigma"].astype(np.float64)
    col = st["ray_col"].astype(np.float64)
    return (col[:, :1] * sig[0][None, :] + col[:, 1:2] * sig[1][None, :]).min(axis=1)


def test_limit_removes_optically_thick_rays():
    inp = W.make_inputs(SPEC)
    off = PT.oracle_states(inp, SEED, SPEC.steps)
    on = PT.oracle_states(inp, SEED, SPEC.steps, tau_max=TAU)
    assert "ray_col" not in off[-1]
    # the set-up is the same; once rays have crossed enough gas the limit removes some
    assert len(on[0]["ray_order"]) == len(off[0]["ray_order"])
    assert len(on[-1]["ray_order"]) < len(off[-1]["ray_order"])
    for s in range(1, SPEC.steps + 1):
        st = on[s]
        assert float(st["tau_max"][0]) == TAU
        col = st["ray_col"]
        assert np.isfinite(col).all() and (col >= 0).all()
        # a live ray that walked this step is below the limit in its most transparent bin
        moved = st["ray_active"].astype(bool)
        assert (_tau_min(st)[moved] <= TAU).all(), s
        # the photon ledger closes with the extra removals (killed photons)
        led = st["ledger"]
        assert led[2] >= 0.0


def test_limit_off_leaves_the_step_unchanged():
    inp = W.make_inputs(SPEC)
    a = PT.oracle_states(inp, SEED, 3)
    b = PT.oracle_states(inp, SEED, 3, tau_max=0.0)
    for x, y in zip(a, b):
        for k in ("ray_order", "ray_geom", "ray_nphot", "nH1", "temp"):
            assert np.array_equal(x[k], y[k]), k
