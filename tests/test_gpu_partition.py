"""One box shared by several contexts, each casting a share of the sources (partition.py), run on
one GPU with the contexts combined in-process between the phases of the step: the shared run must
match the oracle's one-box run with the contract tolerances of tests/test_gpu_parity.py, every
share must hold bit-identical cell state, and the shares' ray totals must add up."""
import numpy as np
import pytest

import parity_tools as PT
from flexrt_imaging_reion_b200 import partition as P, rt, workloads as W
from test_gpu_parity import check

pytestmark = pytest.mark.gpu


def _union_state(shares):
    st = PT.device_state(shares[0], 0, False)
    parts = [PT.device_state(c, 0, False) for c in shares[1:]]
    for k in ("ray_order", "ray_pixel", "ray_itheta", "ray_cell", "ray_geom", "ray_nphot"):
        st[k] = np.concatenate([st[k]] + [p[k] for p in parts])
    # every share runs the same cell passes on the same combined inputs
    for p in parts:
        for k in ("f_H1", "f_He1", "temp", "gamma_H1_tot", "gamma_He1_tot"):
            np.testing.assert_array_equal(p[k], st[k], err_msg=k)
    return st


@pytest.mark.parametrize("case", ["T16x3", "Sx2"])
def test_shares_match_oracle(case):
    if case == "T16x3":
        # a ray capacity below the merge threshold: merging cannot be reached
        spec, seed, world, cap = W.config_tiny(steps=6), 11, 3, 40000
    else:
        spec, seed, world, cap = W.config_S(), 21, 2, 1 << 20
        spec = W.BoxSpec(**{**spec.__dict__, "steps": 4})
    inp = W.make_inputs(spec)
    ref = PT.oracle_states(inp, seed, spec.steps)
    shares = [P.make_share(inp, seed, r, world, ray_capacity=cap) for r in range(world)]
    comb = P.LocalCombiner(shares)
    states = [_union_state(shares)]
    in0 = sum(c.in_flight() for c in shares)
    stats = []
    for s in range(spec.steps):
        tot = P.sum_stats(P.step_shares(shares, comb))
        assert tot["error_flags"] == 0, tot
        assert tot["crossings"] == int(ref[s + 1]["scalars"][10]), (s, tot["crossings"], ref[s + 1]["scalars"][10])
        stats.append(tot)
        states.append(_union_state(shares))
    for c in shares:
        c.close()
    check(states, ref, False)
    assert PT.photon_budget(stats, in0) < 1e-6


@pytest.mark.parametrize("case,world", [("T16M", 2), ("T16N", 3)])
def test_shares_merge_like_one_box(case, world):
    """Boxes whose ray count reaches the merge threshold: in the steps that merge, the shares hand
    their rays to share 0, which merges, splits and compacts them all; the rays are dealt out
    again after the step. Against the oracle's one-box run with the merged-ray tolerances of
    tests/test_gpu_parity.py (merged rays carry float sums in another order), and merging must
    really happen."""
    from test_gpu_parity import T16M, T16N
    spec, seed = {"T16M": T16M, "T16N": T16N}[case]
    inp = W.make_inputs(spec)
    ref = PT.oracle_states(inp, seed, spec.steps)
    shares = [P.make_share(inp, seed, r, world, ray_capacity=1 << 20) for r in range(world)]
    assert P.merge_reachable(shares[0])
    comb = P.LocalCombiner(shares)
    states = [_union_state(shares)]
    in0 = sum(c.in_flight() for c in shares)
    stats = []
    merged = 0
    for s in range(spec.steps):
        tot = P.sum_stats(P.step_shares(shares, comb))
        assert tot["error_flags"] == 0, tot
        assert tot["crossings"] == int(ref[s + 1]["scalars"][10]), (s, tot["crossings"], ref[s + 1]["scalars"][10])
        merged += tot["rays_merged"]
        stats.append(tot)
        states.append(_union_state(shares))
        # every share splits with the same merge threshold, and no share is left without rays
        nm = {c.box_scalars()["nphot_merge"] for c in shares}
        assert len(nm) == 1, nm
    for c in shares:
        c.close()
    check(states, ref, False, merged=True)
    assert merged > 0 and any(float(r["scalars"][4]) > 0 for r in ref)
    assert PT.photon_budget(stats, in0) < 1e-6


def test_one_share_async_phases_match_oracle():
    """The phased step with one share and phases that only enqueue (frt_set_phase_async: no host
    synchronisation between phases, the one-GPU run of bench.py --mode partition) against the
    oracle."""
    spec, seed, cap = W.config_S(), 21, 1 << 20
    spec = W.BoxSpec(**{**spec.__dict__, "steps": 4})
    inp = W.make_inputs(spec)
    ref = PT.oracle_states(inp, seed, spec.steps)
    # a ray capacity below S's merge threshold (2.6e6 rays): the phased step needs it
    ctx = P.make_share(inp, seed, 0, 1, ray_capacity=cap)
    ctx.set_phase_async(True)
    assert ctx.phase_stream() != 0
    comb = P.LocalCombiner([ctx])
    states, stats = [PT.device_state(ctx, 0, False)], []
    for s in range(spec.steps):
        tot = P.step_shares([ctx], comb)[0]
        assert tot["error_flags"] == 0, tot
        assert tot["crossings"] == int(ref[s + 1]["scalars"][10])
        stats.append(tot)
        states.append(PT.device_state(ctx, 0, False))
    ctx.close()
    check(states, ref, False, stats=stats)
