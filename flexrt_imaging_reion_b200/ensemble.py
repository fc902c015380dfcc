"""Uneven ensembles of independent boxes: the batched form (every box in one context, one CUDA
graph per step) against the per-box launch loop, and the sharding of an ensemble across ranks.

The reference runs one box per process (main.cc:108-264 drives the global state of a single
grid), so an ensemble there is a loop of independent runs. Here the boxes share one device
context: one kernel per stage covers the cells and rays of all boxes (each cell and ray carries
its box), and the whole step of all boxes is one graph launch. Boxes never exchange anything, so
across GPUs an ensemble shards by whole boxes with no collective in the step; the per-box totals
are gathered once at the end.
"""
from __future__ import annotations

import time
from typing import Dict, List, Sequence

from . import workloads as W

# Live rays per source of an ensemble box within 10 steps of 0.5 Myr: the oracle's counts over
# the ensemble's boxes are typically 100-250 and peak at 450. The cost model uses the typical
# value, the ray-pool capacity takes the peak with headroom.
RAYS_PER_SOURCE = 250
RAY_SLOTS_PER_SOURCE = 1000


def box_cost(spec: W.BoxSpec, itercount: int = 5) -> float:
    """Relative cost of one step of a box: the cell passes (N^3 per C2Ray iteration) plus the ray
    work (rays per source x sources, each walked once per iteration)."""
    return float(spec.n ** 3 * itercount + spec.n_src * RAYS_PER_SOURCE * (1 + itercount))


def lpt_shards(costs: Sequence[float], nrank: int) -> List[List[int]]:
    """Longest-processing-time packing: boxes in decreasing cost, each to the least-loaded rank
    (ties to the lower rank). Deterministic, so every rank computes the same plan."""
    if nrank < 1:
        raise ValueError("nrank must be >= 1")
    load = [0.0] * nrank
    out: List[List[int]] = [[] for _ in range(nrank)]
    for b in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(nrank), key=lambda k: (load[k], k))
        out[r].append(b)
        load[r] += costs[b]
    for r in out:
        r.sort()
    return out


def ray_capacity(specs: Sequence[W.BoxSpec]) -> int:
    return max(1 << 16, RAY_SLOTS_PER_SOURCE * sum(s.n_src for s in specs))


def _ctx(inputs, seeds, device):
    from .rt import RTContext
    specs = [i.spec for i in inputs]
    return RTContext(inputs, seeds, precision="mixed", outputs="core", ray_capacity=ray_capacity(specs),
                     device=device)


def run_batched(inputs: Sequence[W.BoxInputs], seeds: Sequence[int], warmup: int, steps: int,
                device: int = 0, box_ids: Sequence[int] = (), autotune_steps: int = 0) -> Dict[str, object]:
    """All boxes in one context, one graph launch per step. Device time from CUDA events around
    each graph launch; wall time around the frt_step calls (H2D of the step's random angles,
    launch, D2H of the step totals); raypass_ms sums the CUDA-event time of the ray passes. per_box
    maps each box id to [t, dt, live rays]. With autotune_steps > 0 the last that many warm-up
    steps are frt_autotune's (the chosen launch shapes are returned as "tuning")."""
    ctx = _ctx(inputs, seeds, device)
    ctx.setup()
    n_tune = min(autotune_steps, warmup)
    for _ in range(warmup - n_tune):
        ctx.step(graph=True)
    tuning = ctx.autotune(n_tune) if n_tune else None
    cross, dev_ms, dark_ms, rp_ms, lit = 0, 0.0, 0.0, 0.0, 0
    t0 = time.perf_counter()
    for _ in range(steps):
        st = ctx.step(graph=True)
        cross += st["crossings"]
        lit += st["lit_cells"]
        ms, dms = ctx.last_timing()
        dev_ms += ms
        dark_ms += dms
        rp_ms += ctx.last_raypass_ms()
    wall = time.perf_counter() - t0
    ids = list(box_ids) or list(range(ctx.nbox))
    per_box = {}
    for b in range(ctx.nbox):
        sc = ctx.box_scalars(b)
        per_box[ids[b]] = [sc["t"], sc["dt"], float(ctx.num_rays(b))]
    rays = ctx.num_rays()
    itercount = ctx.itercount
    ctx.close()
    return {"crossings": cross, "device_ms": dev_ms, "dark_ms": dark_ms, "raypass_ms": rp_ms, "lit_cells": lit,
            "wall_s": wall, "rays": rays, "per_box": per_box, "itercount": itercount, "tuning": tuning}


def run_per_box_loop(inputs: Sequence[W.BoxInputs], seeds: Sequence[int], warmup: int, steps: int,
                     device: int = 0, per_source: bool = False) -> Dict[str, float]:
    """The unbatched form: one context per box, every kernel launched directly (no graph), the
    boxes stepped one after another; with per_source, the cast is also one launch per source.
    Timed by host wall clock around each step of all boxes (each plain step ends with a
    synchronising read of its totals)."""
    ctxs = []
    for inp, seed in zip(inputs, seeds):
        c = _ctx([inp], [seed], device)
        c.setup()
        if per_source:
            c.set_cast_per_source(True)
        ctxs.append(c)
    for _ in range(warmup):
        for c in ctxs:
            c.step(graph=False)
    cross = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        for c in ctxs:
            cross += c.step(graph=False)["crossings"]
    wall = time.perf_counter() - t0
    per_box_rays = [float(c.num_rays()) for c in ctxs]
    for c in ctxs:
        c.close()
    return {"crossings": cross, "wall_s": wall, "rays": sum(per_box_rays), "per_box_rays": per_box_rays}


def gather_box_results(local: Dict[int, List[float]], world: int) -> Dict[int, List[float]]:
    """The one exchange of a sharded ensemble: every rank's per-box results, gathered to all
    ranks after the last step (torch.distributed object gather; any backend)."""
    if world == 1:
        return dict(local)
    import torch.distributed as tdist
    parts: List[Dict[int, List[float]]] = [None] * world  # type: ignore[list-item]
    tdist.all_gather_object(parts, local)
    out: Dict[int, List[float]] = {}
    for p in parts:
        for k, v in p.items():
            if k in out:
                raise RuntimeError(f"box {k} reported by two ranks")
            out[k] = v
    return out
