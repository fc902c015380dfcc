"""The autotuner: its search on synthetic costs (CPU, the host-only search compiled alone with
tests/tune_search_test.cc), the shape interface of the C ABI, and on the GPU that the tuned step is
no slower than the default shapes and that other shapes give the same results."""
import os
import subprocess

import numpy as np
import pytest

import parity_tools as PT
from flexrt_imaging_reion_b200 import rt, workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(REPO, "flexrt_imaging_reion_b200", "csrc")


def test_search_finds_optimum(tmp_path):
    exe = str(tmp_path / "tune_search_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", CSRC, os.path.join(HERE, "tune_search_test.cc"),
                    os.path.join(CSRC, "frt_tune.cc"), "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        tok = line.split()
        if tok[0] == "REF":
            opt, start = float(tok[2]), float(tok[3])
            continue
        _, name, rounds, block, grid, chunk, cost = tok
        res[name] = (int(rounds), int(block), int(grid), int(chunk), float(cost))
    # three rounds of four candidates (12 timings of 32 shapes): within 20 % of the optimum's cost
    # and well below the start's; the drifting costs (every round cheaper per unit) end the same
    assert res["separable"][4] <= 1.2 * opt and res["separable"][4] < 0.75 * start, (res, opt, start)
    assert res["drift"][1:4] == res["separable"][1:4], res
    assert res["start_best"][1:3] == (256, 8), res
    assert res["grid_only"][2] == 2, res


def test_set_tuning_rejects_bad_shapes(product_lib):
    import ctypes as C
    from flexrt_imaging_reion_b200 import _abi
    t = _abi.Tuning()   # all zero: invalid
    assert product_lib.frt_set_tuning(None, C.byref(t)) == _abi.FRT_ERR_INVALID


@pytest.mark.gpu
def test_tuned_step_not_slower_than_default():
    """Two contexts of the L box in lockstep (same seed, same steps): one keeps the default shapes,
    the other runs frt_autotune over four of its warm-up steps (two search rounds, then one whole
    graph step with the search's shapes and one with the starting shapes, the faster kept). Then
    both take the same graph steps, alternating, and the tuned one's device time per step is at
    most 2 % above the default's."""
    spec, seed = W.config_L(), 1234
    a = rt.RTContext([W.make_inputs(spec)], [seed], ray_capacity=16 << 20)
    b = rt.RTContext([W.make_inputs(spec)], [seed], ray_capacity=16 << 20)
    a.setup()
    b.setup()
    for _ in range(2):
        a.step()
        b.step()
    for _ in range(4):
        a.step(graph=False)
    tuned = b.autotune(4)
    print("tuned shapes:", tuned)
    ta, tb = [], []
    for _ in range(8):
        sa, sb = a.step(), b.step()
        assert sa["error_flags"] == 0 and sb["error_flags"] == 0
        ta.append(a.last_timing()[0])
        tb.append(b.last_timing()[0])
    ma, mb = float(np.median(ta)), float(np.median(tb))
    print(f"default {ma:.3f} ms/step, tuned {mb:.3f} ms/step")
    a.close()
    b.close()
    assert mb <= 1.02 * ma


@pytest.mark.gpu
@pytest.mark.parametrize("chunk", [32, 512])
def test_other_shapes_same_results(chunk):
    """S with non-default shapes (ray pass as a chunked queue with 128-thread blocks, other grids)
    against the oracle at the contract tolerances."""
    from test_gpu_parity import check
    spec, seed = W.config_S(), 21
    ref = PT.oracle_states(W.make_inputs(spec), seed, spec.steps)
    ctx = rt.RTContext([W.make_inputs(spec)], [seed], outputs="core", ray_capacity=1 << 20)
    ctx.setup()
    ctx.set_tuning(raypass_block=128, raypass_blocks_per_sm=12, raypass_chunk=chunk, walk_block=128,
                   walk_blocks_per_sm=16, cellpass_blocks_per_sm=4, split_blocks_per_sm=2)
    states, stats = [PT.device_state(ctx, 0, False)], []
    for _ in range(spec.steps):
        stats.append(ctx.step())
        states.append(PT.device_state(ctx, 0, False))
    ctx.close()
    check(states, ref, False, stats=stats)


@pytest.mark.gpu
def test_autotune_steps_match_oracle():
    """The tuning steps are real steps: T16 tuned over its first 4 steps (two searched, two
    validating the choice on whole graph steps), then stepped on, matches the oracle at every
    step."""
    from test_gpu_parity import check
    spec, seed = W.config_tiny(), 11
    ref = PT.oracle_states(W.make_inputs(spec), seed, spec.steps)
    ctx = rt.RTContext([W.make_inputs(spec)], [seed], outputs="core", ray_capacity=1 << 20)
    ctx.setup()
    states = [PT.device_state(ctx, 0, False)]
    t = ctx.autotune(4)
    assert t["steps"] == 4
    states += [None] * 4
    states[4] = PT.device_state(ctx, 0, False)
    for _ in range(spec.steps - 4):
        ctx.step()
        states.append(PT.device_state(ctx, 0, False))
    ctx.close()
    check([states[0]] + states[4:], [ref[0]] + ref[4:], False)
