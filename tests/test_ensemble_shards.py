"""Sharding an uneven ensemble across ranks (CPU, gloo): the longest-processing-time plan covers
every box once and balances the load, and a 2-rank run of the plan -- each rank stepping its own
boxes, one gather at the end -- reproduces the one-process run box for box."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as tdist
import torch.multiprocessing as mp

from flexrt_imaging_reion_b200 import ensemble as E, workloads as W


def test_lpt_plan_covers_and_balances():
    specs = W.config_E()
    costs = [E.box_cost(s) for s in specs]
    for nrank in (1, 2, 3, 4, 8):
        plan = E.lpt_shards(costs, nrank)
        flat = sorted(b for r in plan for b in r)
        assert flat == list(range(len(specs)))
        loads = [sum(costs[b] for b in r) for r in plan]
        # Graham's bound for LPT: at most (4/3 - 1/(3m)) of the optimum, which is itself at least
        # max(total / m, largest box)
        opt_lb = max(sum(costs) / nrank, max(costs))
        assert max(loads) <= (4.0 / 3.0 - 1.0 / (3 * nrank)) * opt_lb * (1 + 1e-12)
        assert plan == E.lpt_shards(costs, nrank)   # deterministic: every rank derives the same plan


def test_lpt_plan_edge_cases():
    assert E.lpt_shards([], 3) == [[], [], []]
    assert E.lpt_shards([5.0], 2) == [[0], []]
    assert E.lpt_shards([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        E.lpt_shards([1.0], 0)


SPECS = [W.config_tiny(n=n, n_src=k, steps=3, seed=40 + i, name=f"G{i}")
         for i, (n, k) in enumerate([(8, 2), (12, 3), (16, 4), (10, 2), (12, 1)])]


def _run_boxes(box_ids):
    """Each box stepped alone by the oracle: the CPU stand-in for a rank's batched context."""
    from oracle.oracle import Oracle
    out = {}
    for b in box_ids:
        o = Oracle(W.make_inputs(SPECS[b]), 100 + b)
        for _ in range(SPECS[b].steps):
            o.step()
        out[b] = [float(x) for x in o.scalars()[:8]] + [float(o.num_rays())]
        o.close()
    return out


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        plan = E.lpt_shards([E.box_cost(s) for s in SPECS], world)
        local = _run_boxes(plan[rank])
        allres = E.gather_box_results(local, world)
        q.put((rank, plan[rank], allres))
    finally:
        tdist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_ensemble_two_ranks_matches_one_process():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    single = _run_boxes(range(len(SPECS)))
    owned = sorted(b for _, mine, _ in got for b in mine)
    assert owned == list(range(len(SPECS)))
    for _, _, allres in got:
        assert sorted(allres) == list(range(len(SPECS)))
        for b in range(len(SPECS)):
            np.testing.assert_array_equal(np.array(allres[b]), np.array(single[b]))
