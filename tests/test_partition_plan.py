"""Host side of a box shared by several contexts (CPU): the source shares cover every source
once and balance the luminosity, and the per-context totals add up to the box's."""
import numpy as np
import pytest

from flexrt_imaging_reion_b200 import partition as P, workloads as W


def test_source_shares_cover_and_balance():
    _, lum = W.grid_sources(W.make_inputs(W.config_M()))
    for world in (1, 2, 3, 8):
        masks = P.source_owner_masks(lum, world)
        tot = np.sum(masks, axis=0)
        assert (tot == 1).all()
        counts = [int(m.sum()) for m in masks]
        assert max(counts) - min(counts) <= 1
        share = [float(np.sum(np.asarray(lum)[m == 1])) for m in masks]
        # round robin from the brightest: no share exceeds another by more than the brightest source
        assert max(share) - min(share) <= float(np.max(lum)) * (1 + 1e-12)
    with pytest.raises(ValueError):
        P.source_owner_masks(lum, 0)


def test_sum_stats():
    a = {"rays_alive": 3, "crossings": 10, "lit_cells": 7, "photons_emitted": 1.5, "t": 2.0, "dt": 0.5,
         "error_flags": 0}
    b = {"rays_alive": 4, "crossings": 11, "lit_cells": 7, "photons_emitted": 2.5, "t": 2.0, "dt": 0.5,
         "error_flags": 2}
    s = P.sum_stats([a, b])
    assert s["rays_alive"] == 7 and s["crossings"] == 21 and s["lit_cells"] == 7
    assert s["photons_emitted"] == 4.0 and s["t"] == 2.0 and s["dt"] == 0.5 and s["error_flags"] == 2


class _HostShare:
    """Stands in for a context on the host: each phase writes what its rank would contribute and
    records what the exchange left in the shared arrays."""

    def __init__(self, rank, ncell=64, nlit=8):
        import torch
        self.rank = rank
        self.flags = torch.zeros(ncell, dtype=torch.uint8)
        self.acc = torch.zeros(2 * nlit)
        self.heat = torch.zeros(2 * nlit)
        self.log, self.seen = [], []

    def step_phase(self, phase, it=0):
        from flexrt_imaging_reion_b200 import _abi
        self.log.append((phase, it))
        if phase == _abi.PHASE_WALK:
            self.flags[self.rank::2] = 1
        elif phase == _abi.PHASE_CELLS:
            self.cells_flags = self.flags.clone()
        elif phase == _abi.PHASE_RAYPASS:
            self.acc.fill_(float(self.rank + 1 + it))
            if it == 4:
                self.heat.fill_(10.0 * (self.rank + 1))
        elif phase == _abi.PHASE_CELLPASS:
            self.seen.append((float(self.acc[0]), float(self.heat[0])))
        return {"crossings": self.rank + 1}


def _share_worker(rank, world, port, q):
    import os
    import torch.distributed as tdist
    from flexrt_imaging_reion_b200 import _abi
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        share = _HostShare(rank)
        comb = P.DistCombiner(share, 0, views=lambda c: (c.flags, c.acc, c.heat), sync=lambda: None)
        stats = P.step_shares([share], comb)
        q.put((rank, share.log, bool((share.cells_flags == 1).all()), share.seen, stats))
    finally:
        tdist.destroy_process_group()


def test_two_rank_exchange_over_gloo():
    """The phase order and the exchanges of a box shared by 2 ranks: the lit flags are ORed
    before the cell phase, each ray pass's pairs are summed before its cell pass, the heating
    pairs after the last ray pass."""
    import socket
    import torch.multiprocessing as mp
    from flexrt_imaging_reion_b200 import _abi
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_share_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want_log = [(_abi.PHASE_WALK, 0), (_abi.PHASE_CELLS, 0)]
    for it in range(5):
        want_log += [(_abi.PHASE_RAYPASS, it), (_abi.PHASE_CELLPASS, it)]
    want_log.append((_abi.PHASE_END, 0))
    for rank, log, flags_or, seen, stats in got:
        assert log == want_log
        assert flags_or
        # sums over the ranks: (1 + it) + (2 + it); heating 10 + 20 after the last ray pass
        assert [a for a, _ in seen] == [3.0 + 2 * it for it in range(5)]
        assert seen[-1][1] == 30.0 and all(h == 0.0 for _, h in seen[:-1])
        assert P.sum_stats([st for _, _, _, _, sts in got for st in sts])["crossings"] == 3
