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
    records what the exchange left in the shared arrays. Its rays are ray records (bytes) of F = 5
    bins; with `thresh` set the box can reach its merge threshold."""

    F = 5

    def __init__(self, rank, ncell=64, nlit=8, nrays=0, thresh=None):
        import types
        import torch
        self.rank = rank
        self.flags = torch.zeros(ncell, dtype=torch.uint8)
        self.acc = torch.zeros(2 * nlit)
        self.heat = torch.zeros(2 * nlit)
        self.log, self.seen = [], []
        rec = P.RAY_RECORD_HEAD + 4 * self.F
        self.rays = [bytes([10 * rank + k]) * rec for k in range(nrays)]
        self.thresh = 1 << 40 if thresh is None else thresh
        self._cfg = types.SimpleNamespace(ray_capacity=1 << 30)
        self.nphot_merge = 0.0
        self.end_rays = None

    # the merge exchange's calls
    def box_scalars(self, box=0):
        return {"num_thresh": self.thresh, "nphot_merge": self.nphot_merge}

    def count_rays(self):
        return np.array([len(self.rays)])

    def take_rays(self, box=0, in_step=False):
        data = b"".join(self.rays) + (-1).to_bytes(8, "little", signed=True)
        self.rays = []
        return data

    def put_rays(self, data, box=0):
        rec = P.RAY_RECORD_HEAD + 4 * self.F
        self.rays += [data[k:k + rec] for k in range(0, len(data) - 8, rec)]

    def set_nphot_merge(self, v, box=0):
        self.nphot_merge = v

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
        elif phase == _abi.PHASE_END:
            self.end_rays = sorted(r[0] for r in self.rays)
            if len(self.rays) > self.thresh:   # the merge of this context sets the threshold
                self.nphot_merge = 7.5
        return {"crossings": self.rank + 1}


def _share_worker(rank, world, port, q, merge=False):
    import os
    import torch.distributed as tdist
    from flexrt_imaging_reion_b200 import _abi
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        share = _HostShare(rank, nrays=3 + rank, thresh=6) if merge else _HostShare(rank)
        comb = P.DistCombiner(share, 0, views=lambda c: (c.flags, c.acc, c.heat), sync=lambda: None)
        stats = P.step_shares([share], comb)
        if merge:
            q.put((rank, share.end_rays, sorted(r[0] for r in share.rays), share.nphot_merge))
        else:
            q.put((rank, share.log, bool((share.cells_flags == 1).all()), share.seen, stats))
    finally:
        tdist.destroy_process_group()


def _spawn_ranks(world, merge):
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_share_worker, args=(r, world, port, q, merge)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return got


def test_two_rank_merge_exchange_over_gloo():
    """A box whose rays together exceed its merge threshold (3 + 4 rays against 6): rank 1 hands
    its live rays to rank 0 before the end phase, rank 0 ends the step with all of them and sets
    the merge threshold, which rank 1 takes over, and the rays are dealt out again in order."""
    got = _spawn_ranks(2, True)
    (r0, end0, after0, nm0), (r1, end1, after1, nm1) = got
    assert end0 == [0, 1, 2, 10, 11, 12, 13] and end1 == []
    assert nm0 == nm1 == 7.5
    assert after0 == [0, 1, 2] and after1 == [10, 11, 12, 13]


def test_record_split_keeps_every_ray():
    """split_records deals a record set out in order without losing or duplicating a ray."""
    rec = P.RAY_RECORD_HEAD + 4 * 5
    data = b"".join(bytes([k % 251]) * rec for k in range(10)) + (-1).to_bytes(8, "little", signed=True)
    parts = P.split_records(data, 5, 3)
    assert [(len(p) - 8) // rec for p in parts] == [3, 3, 4]
    assert b"".join(p[:-8] for p in parts) == data[:-8]
    with pytest.raises(ValueError):
        P.split_records(data[:-1], 5, 2)


def test_two_rank_exchange_over_gloo():
    """The phase order and the exchanges of a box shared by 2 ranks: the lit flags are ORed
    before the cell phase, each ray pass's pairs are summed before its cell pass, the heating
    pairs after the last ray pass."""
    from flexrt_imaging_reion_b200 import _abi
    got = _spawn_ranks(2, False)
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
