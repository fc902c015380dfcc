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


def e_subset():
    """One box of the uneven ensemble per grid size (32, 64, 96, 128 cells per side), each the one
    with the most sources of its size; the box with the most sources of the whole ensemble (4005)
    is among them."""
    from flexrt_imaging_reion_b200 import ensemble as EN  # noqa: F401
    specs = W.config_E()
    pick = {}
    for b, s in enumerate(specs):
        if s.n not in pick or s.n_src > specs[pick[s.n]].n_src:
            pick[s.n] = b
    return [(specs[b], 1234 + b) for _, b in sorted(pick.items())]


def test_e_subset_parity():
    """Four real ensemble boxes (32^3 to 128^3, 3546-4005 sources each), batched in one context
    as the benchmark runs them, 3 steps, against one oracle run per box; the step's photon ledger
    of the context against the sum of the boxes' oracle ledgers."""
    from flexrt_imaging_reion_b200 import ensemble as EN
    boxes = e_subset()
    steps = 3
    refs = [PT.oracle_states(W.make_inputs(spec), seed, steps) for spec, seed in boxes]
    inputs = [W.make_inputs(spec) for spec, _ in boxes]
    ctx = rt.RTContext(inputs, [seed for _, seed in boxes], precision="mixed", outputs="core",
                       ray_capacity=EN.ray_capacity([spec for spec, _ in boxes]))
    ctx.setup()
    states = [[PT.device_state(ctx, b, False)] for b in range(len(boxes))]
    stats = []
    for s in range(1, steps + 1):
        st = ctx.step(graph=True)
        assert st["error_flags"] == 0, st
        assert st["crossings"] == sum(int(r[s]["scalars"][10]) for r in refs)
        stats.append(st)
        for b in range(len(boxes)):
            states[b].append(PT.device_state(ctx, b, False))
    ctx.close()
    for b in range(len(boxes)):
        check(states[b], refs[b], False)
    emitted = sum(float(r[0]["ledger"][0]) for r in refs)
    for s in range(1, steps + 1):
        emitted += sum(float(r[s]["ledger"][0]) for r in refs)
        led = {k: 0.0 for k in ("photons_emitted", "photons_deposited", "photons_killed", "photons_overlap",
                                "photons_in_flight")}
        for j, k in enumerate(led):
            led[k] = abs(float(stats[s - 1][k]) - sum(float(r[s]["ledger"][j]) for r in refs)) / emitted
        assert max(led.values()) < 1e-6, (s, led)


def test_e_batched_graph_beats_per_box_loop():
    """The whole uneven ensemble (96 boxes, 32^3-128^3): the batched form (all boxes in one
    context, one graph launch per step) against the per-box loop (one context per box, every
    kernel launched directly, boxes one after another), the same boxes, seeds and steps, both timed
    by host wall clock around the steps. Target: batched at least 3x the loop's crossings/s on the
    same work. The two forms sum a cell's deposits in different orders (other grids, other float
    atomic interleavings), so a ray whose photon count ties with nphot_min, or with a bin edge of a
    box's merge-threshold histogram, can go the other way and change that box's later rays; most
    boxes keep identical ray counts and the crossings agree to 1e-3."""
    from flexrt_imaging_reion_b200 import ensemble as EN
    specs = W.config_E()
    inputs = [W.make_inputs(s) for s in specs]
    seeds = [1234 + b for b in range(len(specs))]
    warmup, steps = 3, 4
    bat = EN.run_batched(inputs, seeds, warmup, steps)
    loop = EN.run_per_box_loop(inputs, seeds, warmup, steps)
    rate_b = bat["crossings"] / bat["wall_s"]
    rate_l = loop["crossings"] / loop["wall_s"]
    print(f"E: batched {rate_b:.3e} crossings/s ({1e3 * bat['wall_s'] / steps:.2f} ms/step), per-box loop "
          f"{rate_l:.3e} ({1e3 * loop['wall_s'] / steps:.2f} ms/step), ratio {rate_b / rate_l:.2f}")
    same = sum(1 for b in range(len(specs)) if bat["per_box"][b][2] == loop["per_box_rays"][b])
    print(f"E: crossings batched {bat['crossings']} loop {loop['crossings']}; boxes with identical live rays "
          f"{same} of {len(specs)}")
    assert abs(bat["crossings"] - loop["crossings"]) <= 1e-3 * bat["crossings"]
    assert same >= 0.9 * len(specs)
    assert rate_b >= 3.0 * rate_l
