"""One box over several contexts: a share of its sources per context (per GPU).

Rays of different sources meet only through the photo-ionisation rates of the cells they cross,
so a box whose ray count cannot reach the merge threshold (merging is the one step that combines
rays of different sources) splits exactly by sources. Every context holds the whole box and casts
only its sources (frt_set_source_owner); the step runs in phases (frt_step_phase) and, between
them, the contexts combine two things:

* after the walk, the lit-cell flags (OR over the contexts, one byte per cell), so that every
  context numbers the same lit cells in the same order;
* after each of the 5 ray passes, the lit cells' absorbed photons (a sum of float2 pairs), and
  after the last one also the photo-heating pairs.

Every context then runs the same cell passes and holds the same cell state; the ray-side work
(walk, ray passes, compaction, splitting, cast) is divided by the number of contexts. The sums
of the float pairs are taken in a different order than one context's atomics take them, so the
results agree with a one-context run to float rounding (and the ray trees agree up to rays whose
photon count ties with nphot_min).

A box whose ray count reaches its merge threshold merges rays of different sources, so in a step
where the contexts' live rays together exceed the threshold (their counts summed after the last
ray pass) the rays are brought together first: every other context hands its live rays to context
0 (frt_take_rays / frt_put_rays, ray records in the reference's ray-file format), context 0 runs
the end of the step (count, merge, split, compaction) on all of them, the others end the step
without rays, context 0's merge threshold nphot_merge goes to the others, and after the step the
rays are dealt out again in equal shares (a ray's context does not matter: every context adds the
deposits of all of them). The records pass through the host: a correct first form whose cost
grows with the ray count of the merging steps.

`DistCombiner` combines over torch.distributed ranks (NCCL, one GPU per rank); `LocalCombiner`
combines contexts that live in one process (the emulation the tests use on one GPU).
"""
from __future__ import annotations

from typing import Dict, List, Sequence

import numpy as np

from . import _abi, rt, workloads as W


def source_owner_masks(lum: Sequence[float], world: int) -> List[np.ndarray]:
    """Owner masks that deal the sources out by luminosity, brightest first, round robin (bright
    sources keep their rays longest): mask r has a 1 for every source of rank r."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = np.argsort(-np.asarray(lum, np.float64), kind="stable")
    masks = [np.zeros(len(lum), np.uint8) for _ in range(world)]
    for k, s in enumerate(order):
        masks[k % world][s] = 1
    return masks


# bytes of a ray record besides its photon counts (frt_write_rays: slot, active flag, order, pixel,
# angle index, direction, r, dr, x, y, z, time, cell); a record set ends with the slot -1
RAY_RECORD_HEAD = 8 + 1 + 2 + 4 + 2 + 12 + 24 + 4
_RECORDS_END = (-1).to_bytes(8, "little", signed=True)


def split_records(data: bytes, nfreq: int, parts: int) -> List[bytes]:
    """A record set cut into `parts` record sets of (nearly) equal ray counts, in order."""
    rec = RAY_RECORD_HEAD + 4 * nfreq
    n = (len(data) - 8) // rec
    if n * rec + 8 != len(data) or data[-8:] != _RECORDS_END:
        raise ValueError("not a ray record set of this frequency count")
    return [data[(n * k // parts) * rec:(n * (k + 1) // parts) * rec] + _RECORDS_END for k in range(parts)]


def merge_reachable(ctx: rt.RTContext) -> bool:
    """Whether the box's ray count can reach its merge threshold with this ray capacity (fixed for
    the context: asked once)."""
    v = getattr(ctx, "_merge_reachable", None)
    if v is None:
        v = ctx.box_scalars()["num_thresh"] < ctx._cfg.ray_capacity
        ctx._merge_reachable = v
    return v


class _DevArray:
    """A device array handed to torch by __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2}


def _views(ctx: rt.RTContext, device: int):
    import torch
    lf, nc, la, lh, nl = ctx.phase_buffers()
    dev = torch.device("cuda", device)
    flags = torch.as_tensor(_DevArray(lf, nc, "|u1"), device=dev)
    acc = torch.as_tensor(_DevArray(la, 2 * nl, "<f4"), device=dev) if nl else None
    heat = torch.as_tensor(_DevArray(lh, 2 * nl, "<f4"), device=dev) if nl else None
    return flags, acc, heat


class LocalCombiner:
    """Combines contexts of one process (all on one device). With one context there is nothing to
    combine, so no work and no synchronisation (the one-GPU run of the phased step)."""

    def __init__(self, ctxs: Sequence[rt.RTContext], device: int = 0):
        self.ctxs, self.device = list(ctxs), device

    def _apply(self, pick, reduce):
        import torch
        if len(self.ctxs) == 1:
            return
        views = [pick(_views(c, self.device)) for c in self.ctxs]
        if views[0] is None:
            return
        tot = views[0].clone()
        for v in views[1:]:
            tot = reduce(tot, v)
        for v in views:
            v.copy_(tot)
        torch.cuda.synchronize(self.device)

    def flags(self):
        import torch
        self._apply(lambda v: v[0], torch.maximum)

    def acc(self):
        self._apply(lambda v: v[1], lambda a, b: a + b)

    def heat(self):
        self._apply(lambda v: v[2], lambda a, b: a + b)

    # the merge of a shared box (see the module docstring)
    def live_rays(self) -> int:
        return sum(int(c.count_rays()[0]) for c in self.ctxs)

    def gather_rays(self):
        for c in self.ctxs[1:]:
            self.ctxs[0].put_rays(c.take_rays(0, in_step=True))

    def share_merge_threshold(self):
        v = self.ctxs[0].box_scalars()["nphot_merge"]
        for c in self.ctxs[1:]:
            c.set_nphot_merge(v)

    def deal_rays(self):
        parts = split_records(self.ctxs[0].take_rays(0, in_step=False), self.ctxs[0].F, len(self.ctxs))
        for c, p in zip(self.ctxs, parts):
            c.put_rays(p)


class DistCombiner:
    """Combines one context per rank over torch.distributed (NCCL: one GPU per rank). `views`
    and `sync` default to the context's device arrays and a device synchronisation; they are
    parameters so that the exchange can be exercised with host tensors over gloo. With
    `on_stream` (the default on a GPU), the context's phases only enqueue and every all-reduce is
    ordered on the context's own stream (torch waits for the phases queued before it and the
    phases queued after it wait for the collective): no host synchronisation between phases."""

    def __init__(self, ctx, device: int, views=None, sync=None, on_stream: bool = None):
        self.ctxs, self.device = [ctx], device
        self._views = views or (lambda c: _views(c, self.device))
        self.on_stream = (views is None and sync is None) if on_stream is None else on_stream
        self._sync = sync or self._device_sync
        self._stream = None
        if self.on_stream:
            import torch
            ctx.set_phase_async(True)
            self._stream = torch.cuda.ExternalStream(ctx.phase_stream(), device=torch.device("cuda", device))

    def _device_sync(self):
        import torch
        torch.cuda.synchronize(self.device)

    def _all_reduce(self, t, op):
        import torch.distributed as dist
        if t is None:
            return
        if self._stream is not None:
            import torch
            with torch.cuda.stream(self._stream):
                dist.all_reduce(t, op=op)
            return
        self._sync()
        dist.all_reduce(t, op=op)
        self._sync()

    def flags(self):
        import torch.distributed as dist
        self._all_reduce(self._views(self.ctxs[0])[0], dist.ReduceOp.MAX)

    def acc(self):
        import torch.distributed as dist
        self._all_reduce(self._views(self.ctxs[0])[1], dist.ReduceOp.SUM)

    def heat(self):
        import torch.distributed as dist
        self._all_reduce(self._views(self.ctxs[0])[2], dist.ReduceOp.SUM)

    # the merge of a shared box: host records through object collectives (every rank takes the
    # same steps in the same order)
    def live_rays(self) -> int:
        import torch.distributed as dist
        out = [None] * dist.get_world_size()
        dist.all_gather_object(out, int(self.ctxs[0].count_rays()[0]))
        return sum(out)

    def gather_rays(self):
        import torch.distributed as dist
        rank, world = dist.get_rank(), dist.get_world_size()
        mine = self.ctxs[0].take_rays(0, in_step=True) if rank != 0 else b""
        got = [None] * world if rank == 0 else None
        dist.gather_object(mine, got, dst=0)
        if rank == 0:
            for data in got[1:]:
                self.ctxs[0].put_rays(data)

    def share_merge_threshold(self):
        import torch.distributed as dist
        v = [self.ctxs[0].box_scalars()["nphot_merge"] if dist.get_rank() == 0 else None]
        dist.broadcast_object_list(v, src=0)
        if dist.get_rank() != 0:
            self.ctxs[0].set_nphot_merge(v[0])

    def deal_rays(self):
        import torch.distributed as dist
        rank, world = dist.get_rank(), dist.get_world_size()
        parts = None
        if rank == 0:
            parts = split_records(self.ctxs[0].take_rays(0, in_step=False), self.ctxs[0].F, world)
        out = [None]
        dist.scatter_object_list(out, parts, src=0)
        self.ctxs[0].put_rays(out[0])


def step_shares(ctxs: Sequence[rt.RTContext], combiner, itercount: int = 5) -> List[Dict[str, float]]:
    """One step of a box shared by `ctxs` (the contexts of this process: all of them for a
    LocalCombiner, this rank's one for a DistCombiner). Returns each context's totals."""
    for c in ctxs:
        c.step_phase(_abi.PHASE_WALK)
    combiner.flags()
    for c in ctxs:
        c.step_phase(_abi.PHASE_CELLS)
    for it in range(itercount):
        for c in ctxs:
            c.step_phase(_abi.PHASE_RAYPASS, it)
        combiner.acc()
        if it == itercount - 1:
            combiner.heat()
        for c in ctxs:
            c.step_phase(_abi.PHASE_CELLPASS, it)
    # a box that can reach its merge threshold: the contexts' live rays counted together, and
    # merged on context 0 when they exceed it
    merge = merge_reachable(ctxs[0]) and combiner.live_rays() > ctxs[0].box_scalars()["num_thresh"]
    if merge:
        combiner.gather_rays()
    stats = [c.step_phase(_abi.PHASE_END) for c in ctxs]
    if merge:
        combiner.share_merge_threshold()
        combiner.deal_rays()
    return stats


def sum_stats(stats: Sequence[Dict[str, float]]) -> Dict[str, float]:
    """Whole-box totals of a step from the contexts' totals (t and dt are the box's)."""
    out = dict(stats[0])
    for k in out:
        if k in ("t", "dt"):
            continue
        if k == "error_flags":
            v = 0
            for st in stats:
                v |= int(st[k])
            out[k] = v
        elif k == "lit_cells":
            out[k] = stats[0][k]   # the same lit list in every context
        else:
            out[k] = sum(st[k] for st in stats)
    return out


def make_share(inp: W.BoxInputs, seed: int, rank: int, world: int, device: int = 0,
               ray_capacity: int = 16 << 20) -> rt.RTContext:
    """The context of share `rank` of `world`: the whole box, its own sources cast."""
    _, lum = W.grid_sources(inp)
    own = source_owner_masks(lum, world)[rank]
    ctx = rt.RTContext([inp], [seed], precision="mixed", outputs="core", ray_capacity=ray_capacity, device=device)
    ctx.setup(owner=own)
    return ctx
