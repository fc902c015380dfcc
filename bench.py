#!/usr/bin/env python
"""Benchmark of the B200 RT step: ray-cell crossings/s and ms per RT step.

Workload (default "L"): the large configuration -- 256^3 box of 100 h^-1 cMpc at z = 6.5,
lognormal gas (sigma_ln = 0.8), 16384 sources with dN/dL ~ L^-2 on [1e50, 1e54] ph/s, 5 frequency
bins, dt = 0.25 Myr -- from seeded synthetic inputs. A "step" is one whole RT step (advance,
5-iteration C2Ray with Gamma deposition, merge, split, thermal, cast); W warm-up steps, then K
timed steps of the same run. The state (16.8 M cells, ~7 M rays) is far larger than L2, so no
L2 flush is needed between steps.

  value      crossings of the K steps / device time of the K steps (CUDA events around each
             graph launch on the step stream), summed over ranks / max over ranks
  e2e        same crossings / host wall time of the frt_step calls (per step: H2D of the step's
             random-angle indices from pinned memory, graph launch, D2H of the step totals)
  roofline   the ray pass (k_raypass_mixed, five launches per step): algorithmic bytes = crossings
             x 84 B / its CUDA-event time, against MEASURED_PEAKS.json hbm_gbs; "walk" gives the
             same for the walk (k_advance) and "dark_pass" the dark-cell pass's span
  cpu_baseline  the reference's own OpenMP code (compiled from its sources, oracle/_ref) on the
             host cores, on a bounded steady-state sample of the same workload: the device's state
             after the last timed step, written in the reference's restart formats, is read by the
             reference's own restart path (input_grid = TRUE), its balance_cpus spreads the rays
             over the threads, and it then runs three timed steps

--impl reference runs that compiled reference alone (all host threads) and prints its line.
Multi-GPU: the single-box workloads do not shard; --gpus N runs N independent replicas (one per
rank, "weak" scaling), value = all ranks' crossings / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import resource
import subprocess
import sys
import tempfile
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

DARK_BYTES_PER_CELL = 82  # 10 float fields + treion_flag + lit_flag read, 10 float fields written
# DRAM bytes per dark cell of one k_dark launch, from ncu (dram__bytes_read.sum + write.sum) at
# step 24 of the L workload: 1344.7 MB for 13 264 001 dark cells. The
# bench scales it by the dark cells of its own steps (traffic grows with the cells processed).
DARK_TRAFFIC_BYTES_PER_CELL = 1344697856 / 13264001
# Ray pass (the dominant kernel): the algorithmic bytes of one crossing in one C2Ray iteration as
# the hot-path analysis counts them -- 8 B segment read, 8 B of gathered <n_HI>, <n_HeI>, 68 B of
# deposits (2 + 3 x 5 floats) -- and the ncu DRAM bytes (read + write) per crossing of one launch,
# the mean over the 5 passes of step 24 of L (17 465 922 crossings per pass; 675.7 MB per launch).
# The number of ray passes per step is the context's C2Ray iteration count (RTContext.itercount).
RAYPASS_BYTES_PER_CROSSING = 8 + 8 + 68
# warm-up steps that frt_autotune takes (the last ones of the warm-up)
AUTOTUNE_STEPS = 4
RAYPASS_TRAFFIC_BYTES_PER_CROSSING = 38.7
# Walk (k_advance): per live ray its record read (cell, geometry, box, time: 44 B) and written
# back with its removal flag (29 B); per moved ray the 16-byte header of the ray passes; per
# crossing its packed segment {cell, dist} written (8 B) and the cell's lit mark (1 B).
WALK_BYTES_PER_RAY = 44 + 29
WALK_BYTES_PER_MOVED = 16
WALK_BYTES_PER_CROSSING = 8 + 1


def _peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of this rank's GPU, sampled during the timed
    region. NVML is polled every 10 ms on the device's UUID (the timed region of the default run
    is a fraction of a second, shorter than one nvidia-smi call); nvidia-smi on the same UUID
    every 200 ms is the fallback. Only reads: no setting of the GPU is changed."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, index: int):
        self.index = index
        self.rows = []          # (sm_mhz, sm_max_mhz, reason bits)
        self.source = None
        self._stop = threading.Event()
        self._t = None

    def _uuid(self):
        try:
            import torch
            u = str(torch.cuda.get_device_properties(self.index).uuid)
            return u if u.startswith("GPU-") else "GPU-" + u
        except Exception:
            return None

    def _run_nvml(self, uuid):
        import pynvml
        pynvml.nvmlInit()
        try:
            h = (pynvml.nvmlDeviceGetHandleByUUID(uuid.encode()) if uuid
                 else pynvml.nvmlDeviceGetHandleByIndex(self.index))
            get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons",
                                  getattr(pynvml, "nvmlDeviceGetCurrentClocksThrottleReasons", None))
            mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.source = "nvml, 10 ms"
            while not self._stop.is_set():
                sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                bits = int(get_reasons(h)) if get_reasons else 0
                self.rows.append((sm, mx, bits))
                self._stop.wait(0.01)
        finally:
            pynvml.nvmlShutdown()

    def _run_smi(self, uuid):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        self.source = "nvidia-smi, 200 ms"
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={uuid or self.index}", f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                r = [x.strip() for x in out.split(",")]
                if len(r) == 6 and r[0].replace(".", "").isdigit():
                    bits = sum(b for (_, b), v in zip(self.REASONS, r[2:]) if v == "Active")
                    self.rows.append((float(r[0]), float(r[1]), bits))
            except Exception:
                pass
            self._stop.wait(0.2)

    def start(self):
        uuid = self._uuid()

        def run():
            try:
                self._run_nvml(uuid)
            except Exception:
                if not self._stop.is_set():
                    self._run_smi(uuid)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [r[0] for r in self.rows]
        mx = [r[1] for r in self.rows]
        reasons = sorted({n for r in self.rows for n, b in self.REASONS if r[2] & b})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows), "source": self.source}


def _spec(name):
    from flexrt_imaging_reion_b200 import workloads as W
    return {"L": W.config_L, "M": W.config_M, "S": W.config_S}[name]()


def _describe_ensemble(specs):
    sizes = sorted({s.n for s in specs})
    return (f"E: {len(specs)} independent boxes, N in {sizes} (same comoving cell), z={specs[0].z:g}, "
            f"sigma_ln U[0.3,0.9], {sum(s.n_src for s in specs)} sources (log-uniform 8..4096 per box, "
            f"L^-2 [1e50,1e54] ph/s), 5 bins, dt={specs[0].dt_myr} Myr, "
            f"{sum(s.n ** 3 for s in specs) / 1e6:.1f} M cells")


def _describe(spec):
    return (f"{spec.name}: {spec.n}^3, {spec.box_hmpc:g} h^-1 cMpc, z={spec.z:g}, sigma_ln={spec.sigma_ln}, "
            f"{spec.n_src} sources ({spec.lum_law} [{spec.lum_min:.0e},{spec.lum_max:.0e}] ph/s), 5 bins, "
            f"dt={spec.dt_myr} Myr, clumping={spec.clump_model}")


def _unlimited_stack():
    # update_thermal keeps a float[Nx][Ny][Nz] array on the stack (gas_funcs.cc:364)
    try:
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        soft, hard = resource.getrlimit(resource.RLIMIT_STACK)
        resource.setrlimit(resource.RLIMIT_STACK, (hard, hard))


# ---- the compiled reference (oracle/_ref) ------------------------------------------------------
def _ref_exe(name: str, spec, threads: int, restart: bool = False) -> str:
    from oracle import build_ref as B
    d = os.path.join(B.OUT, name)
    exe = os.path.join(d, "ref_driver")
    meta_p = os.path.join(d, "stage.json")
    ncpu = None
    if os.path.exists(meta_p):
        with open(meta_p) as f:
            ncpu = json.load(f).get("ncpu")
    drv = os.path.join(HERE, "oracle", "ref_driver.cc")
    stale = os.path.exists(exe) and os.path.getmtime(exe) < os.path.getmtime(drv)
    if not os.path.exists(exe) or ncpu is None or ncpu < threads or stale:
        if os.path.isdir(B.REF_SRC):
            B.build(name, spec, ncpu=threads, restart=restart)
        elif os.path.isdir(os.path.join(d, "src")):
            B.compile_stage(d, ncpu=threads)
        else:
            raise RuntimeError("compiled reference not available (oracle/_ref/%s)" % name)
    return exe


def run_reference(spec, name: str, steps: int, threads: int, time_cap_s: float, seed: int):
    """Run the compiled reference for up to `steps` steps (stopping once the steps so far exceed
    time_cap_s); returns per-step (crossings, wall) and the set-up time."""
    from flexrt_imaging_reion_b200 import workloads as W
    exe = _ref_exe(name, spec, threads)
    inp = W.make_inputs(spec)
    with tempfile.TemporaryDirectory() as td:
        W.write_reference_inputs(inp, td)
        args = [exe, td, str(steps), str(seed), "0", repr(spec.rkill_cm())]
        if inp.clump is not None:
            args.append(os.path.join(td, "clump.bin"))
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        p = subprocess.Popen(args, cwd=os.path.dirname(exe), env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                             text=True, preexec_fn=_unlimited_stack)
        rows, setup = [], None
        t_steps = 0.0
        for line in p.stdout:
            if line.startswith("SETUP"):
                setup = float(line.split()[1])
            m = re.match(r"STEP (\d+) rays_before=\d+ crossings=(\d+) moved=\d+ wall=([0-9.eE+-]+)", line)
            if m:
                rows.append((int(m.group(2)), float(m.group(3))))
                t_steps += float(m.group(3))
                if t_steps > time_cap_s:
                    p.kill()
                    break
        p.wait()
    return rows, setup


def _step_phases(line: str) -> dict:
    """The key=value fields of one STEP line of the reference driver (step wall time and its parts:
    adv, iter, merge, split, thermal, cast, in s; rays_before, crossings, moved)."""
    out = {}
    for tok in line.split()[2:]:
        k, _, v = tok.partition("=")
        try:
            out[k] = float(v)
        except ValueError:
            pass
    return out


def run_reference_restart(spec, name: str, files, steps: int, threads: int, seed: int):
    """The compiled reference started through its own restart path (input_grid = TRUE: init()
    reads the gas and treion records, init_rt() the ray records, rt_funcs.cc:95-124) from
    `files` = (gas, rays, treion) bytes in its formats, then run for `steps` steps; returns
    per-step (crossings, wall) and the restart set-up time."""
    from flexrt_imaging_reion_b200 import workloads as W
    exe = _ref_exe(name, spec, threads, restart=True)
    d = os.path.dirname(exe)
    gas, rays, tre = files
    paths = [os.path.join(d, "input_files", f"restart_{k}.bin") for k in ("gas", "rays", "tre")]
    try:
        for pth, data in zip(paths, (gas, rays, tre)):
            with open(pth, "wb") as f:
                f.write(data)
        inp = W.make_inputs(spec)
        with tempfile.TemporaryDirectory() as td:
            W.write_reference_inputs(inp, td)
            args = [exe, td, str(steps), str(seed), "0", repr(spec.rkill_cm())]
            # the rays read from the restart file are spread over the threads by the reference's
            # balance_cpus before the first timed step (its step loop does that after every step)
            env = dict(os.environ, OMP_NUM_THREADS=str(threads), FRT_RESTART_BALANCE="1")
            r = subprocess.run(args, cwd=d, env=env, capture_output=True, text=True, preexec_fn=_unlimited_stack)
            if r.returncode != 0:
                raise RuntimeError(f"ref_driver (restart) failed: {r.stdout[-500:]} {r.stderr[-500:]}")
        rows, setup = [], None
        for line in r.stdout.splitlines():
            if line.startswith("SETUP"):
                setup = float(line.split()[1])
            m = re.match(r"STEP (\d+) rays_before=\d+ crossings=(\d+) moved=\d+ wall=([0-9.eE+-]+)", line)
            if m:
                rows.append((int(m.group(2)), float(m.group(3)), _step_phases(line)))
        return rows, setup
    finally:
        for pth in paths:
            if os.path.exists(pth):
                os.remove(pth)


# ---- uneven ensemble (E) --------------------------------------------------------------------
def run_reference_ensemble(steps: int, threads: int, time_cap_s: float, seed: int):
    """The compiled reference over the ensemble's boxes in order (one build per grid size), each
    box for `steps` steps, until the summed step time passes time_cap_s. Returns (crossings,
    step seconds, boxes run)."""
    from flexrt_imaging_reion_b200 import workloads as W
    specs = W.config_E()
    cross, wall, nb = 0, 0.0, 0
    for b, spec in enumerate(specs):
        rows, _ = run_reference(spec, f"E{spec.n}", steps, threads, max(1.0, time_cap_s - wall), seed + b)
        cross += sum(c for c, _ in rows)
        wall += sum(w for _, w in rows)
        nb += 1
        if wall > time_cap_s:
            break
    return cross, wall, nb


def run_ensemble(args, rank: int, world: int, local_rank: int):
    """Batched + graph form of the ensemble (every box of this rank in one context), and on one GPU
    also the per-box launch loop over the same boxes and seeds for the comparison. Across ranks the
    boxes are sharded by the longest-processing-time plan (no exchange inside the step)."""
    from flexrt_imaging_reion_b200 import ensemble as EN, workloads as W
    specs = W.config_E()
    plan = EN.lpt_shards([EN.box_cost(s) for s in specs], world)
    mine = plan[rank]
    inputs = [W.make_inputs(specs[b]) for b in mine]
    seeds = [args.seed + b for b in mine]
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    n_tune = AUTOTUNE_STEPS if (not args.no_autotune and args.subgrid == "off"
                                and args.warmup >= AUTOTUNE_STEPS + 1) else 0
    bat = EN.run_batched(inputs, seeds, args.warmup, args.steps, device=local_rank, box_ids=mine,
                         autotune_steps=n_tune)
    clk = clocks.stop()
    per_box = EN.gather_box_results(bat["per_box"], world)
    ncell = sum(s.n ** 3 for s in (specs[b] for b in mine))
    if dist:
        import torch
        import torch.distributed as tdist
        t = torch.tensor([bat["device_ms"], bat["wall_s"], float(bat["crossings"])], dtype=torch.float64,
                         device=f"cuda:{local_rank}")
        mx, sm = t.clone(), t.clone()
        tdist.all_reduce(mx, op=tdist.ReduceOp.MAX)
        tdist.all_reduce(sm, op=tdist.ReduceOp.SUM)
        dev_ms, wall, cross = float(mx[0]), float(mx[1]), float(sm[2])
    else:
        dev_ms, wall, cross = bat["device_ms"], bat["wall_s"], float(bat["crossings"])
    cap = EN.ray_capacity([specs[b] for b in mine])
    itercount = int(bat["itercount"])
    per_step = max(launches_per_step(specs[b], cap, itercount) for b in mine) if mine else 0
    rp_gbs = (RAYPASS_BYTES_PER_CROSSING * float(bat["crossings"]) * itercount / (bat["raypass_ms"] * 1e-3) / 1e9
              if bat["raypass_ms"] > 0 else None)
    peak, peak_kind = _peaks()
    res = {
        "metric": "ray-cell crossings/s", "value": cross / (dev_ms * 1e-3), "unit": "crossings/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded lognormal gas + L^-2 sources per box)",
        "config": {"workload": _describe_ensemble(specs), "timed_steps": f"{args.warmup + 1}..{args.warmup + args.steps}",
                   "graph": True, "l2": "state larger than L2, no flush",
                   "parallelism": f"boxes sharded over {world} ranks (LPT)" if dist else "single",
                   "launch_shapes": _tuning_config(bat.get("tuning"))},
        "e2e": {"value": cross / wall, "unit": "crossings/s", "h2d_bytes_per_step": 2 * len(mine) + 2 * sum(
            len(W.grid_sources(i)[1]) for i in inputs), "d2h_bytes_per_step": 144},
        # the ray pass (five launches per step on the main stream), as for a single box
        "roofline": {"bound": "hbm", "kernel": "k_raypass_mixed (ray pass of one C2Ray iteration)",
                     "achieved": rp_gbs, "peak": peak, "unit": "GB/s",
                     "frac": (rp_gbs / peak) if rp_gbs else None,
                     "traffic": RAYPASS_TRAFFIC_BYTES_PER_CROSSING * float(bat["crossings"]) / args.steps,
                     "traffic_note": "bytes per launch: ncu DRAM bytes per crossing of a ray pass (L) x crossings per step",
                     "algorithmic_bytes_per_launch": RAYPASS_BYTES_PER_CROSSING * float(bat["crossings"]) / args.steps,
                     "bytes_per_crossing": RAYPASS_BYTES_PER_CROSSING, "peak_kind": peak_kind,
                     "launch_ms": bat["raypass_ms"] / args.steps / itercount, "launches_per_step": itercount},
        "dark_pass": {"kernel": "k_dark (cells no ray touched: whole step in one pass)",
                      "span_ms_per_step": bat["dark_ms"] / args.steps, "bytes_per_cell": DARK_BYTES_PER_CELL,
                      "cells_per_step": ncell - bat["lit_cells"] / args.steps,
                      "note": "CUDA-event span on its own stream; its short blocks run in the gaps of the "
                              "higher-priority lit-cell chain, so the span is not its busy time"},
        "gpu_launches": per_step * args.steps,
        "clocks": clk,
        "crossings_per_step": cross / args.steps,
        "rays_end": sum(v[2] for v in per_box.values()),
    }
    if not dist and not args.no_loop:
        loop = EN.run_per_box_loop(inputs, seeds, args.warmup, args.steps, device=local_rank)
        res["per_box_plain_loop"] = {
            "value": loop["crossings"] / loop["wall_s"], "unit": "crossings/s", "ms_per_step": 1e3 * loop["wall_s"] / args.steps,
            "crossings": loop["crossings"],
            "gpu_launches": args.steps * sum(launches_per_step(specs[b], EN.ray_capacity([specs[b]]), itercount)
                                             for b in mine),
            "what": "one context per box, every kernel launched directly (no graph), boxes one after another; "
                    "host wall clock"}
        res["batched_vs_loop_wall"] = (cross / wall) / (loop["crossings"] / loop["wall_s"])
        # the ray trees agree up to rays whose photon count ties with a threshold (float sums in
        # another order)
        res["crossings_rel_diff"] = abs(loop["crossings"] - bat["crossings"]) / max(1, bat["crossings"])
        ps = EN.run_per_box_loop(inputs, seeds, args.warmup, args.steps, device=local_rank, per_source=True)
        res["per_box_per_source_loop"] = {
            "value": ps["crossings"] / ps["wall_s"], "unit": "crossings/s", "ms_per_step": 1e3 * ps["wall_s"] / args.steps,
            "crossings": ps["crossings"],
            "gpu_launches": args.steps * sum(launches_per_step(specs[b], EN.ray_capacity([specs[b]]), itercount) - 1 +
                                             len(W.grid_sources(inp)[1]) for b, inp in zip(mine, inputs)),
            "what": "as per_box_plain_loop, and the cast launched once per source; host wall clock"}
        res["batched_vs_per_source_loop_wall"] = (cross / wall) / (ps["crossings"] / ps["wall_s"])
    return res


# ---- adjoint (A) ------------------------------------------------------------------------------
def run_adjoint(args):
    """One forward step of the adjoint box (graph, CUDA-event device time) against frt_adjoint of
    the same set-up state (CUDA-event device time of its kernels; the host wall time of the whole
    call, gradient read-back included, is reported beside it)."""
    import numpy as np
    from flexrt_imaging_reion_b200 import workloads as W, rt
    spec = W.config_A()
    inp = W.make_inputs(spec)
    lo, hi = [56, 56, 56], [72, 72, 72]
    fwd = []
    for _ in range(max(3, args.steps)):
        with rt.RTContext([inp], [args.seed], ray_capacity=1 << 20) as c:
            c.setup()
            c.step()
            fwd.append(c.last_timing()[0])
    with rt.RTContext([inp], [args.seed], ray_capacity=1 << 20) as c:
        c.setup()
        for _ in range(args.warmup):
            c.adjoint(lo, hi)
        ts, dev = [], []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            J, dl, dnh = c.adjoint(lo, hi)
            ts.append(1e3 * (time.perf_counter() - t0))
            dev.append(c.last_adjoint_ms())
    step_ms = float(np.median(fwd))
    adj_ms = float(np.median(dev))
    return {"metric": "adjoint cost / forward step (device time)", "value": adj_ms / step_ms, "unit": "ratio",
            "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "step_ms": step_ms, "adjoint_ms": adj_ms, "adjoint_call_ms_wall": float(np.median(ts)),
            "J": J, "nonzero_dnH": int(np.count_nonzero(dnh)),
            "config": {"workload": "A: 128^3, 50 h^-1 cMpc, z=7, 256 sources log-uniform [1e51,1e53] in the centred "
                                   "32^3 cells, 1 step of 1 Myr; J = sum Gamma_HI over the centred 16^3 cells"},
            "dtype": "f64 (adjoint), f32 (forward step)", "data": "synthetic"}


# ---- our arm ---------------------------------------------------------------------------------
def launches_per_step(spec, ray_capacity, itercount=5, hpx_lvl=0):
    """Kernels one fused step launches: clear_lit, step_begin, advance, lit_compact, pk_slots,
    dark, lit_init, itercount x (ray pass + lit pass), the split thresholds (when the pool can
    reach the merge threshold also count and 2 merge set-up kernels before them and 4 binning
    kernels after them), compact_split, swap, the cast's count and scan of the new rays'
    positions, cast."""
    n = 1 + 1 + 1 + 1 + 1 + 1 + 1 + 2 * itercount + 1 + 2 + 3
    num_thresh = (spec.ray_per_cell_max - 12 * 4 ** hpx_lvl) * spec.n ** 3
    if num_thresh < ray_capacity:
        n += 3 + 4
    return n


def run_partition(args, rank: int, world: int, local_rank: int):
    """One box, its sources shared over the ranks (partition.py): every rank holds the whole box,
    walks its share of the rays and runs the same cell passes; per step one OR all-reduce of the
    lit flags and per C2Ray iteration one sum all-reduce of the lit cells' rates (NCCL). Timed by
    CUDA events on the rank's device around each step (collectives included), max over ranks."""
    import torch
    from flexrt_imaging_reion_b200 import partition as P, workloads as W
    spec = _spec(args.workload)
    inp = W.make_inputs(spec)
    ctx = P.make_share(inp, args.seed, rank, world, device=local_rank, ray_capacity=args.ray_capacity)
    if world > 1:
        comb = P.DistCombiner(ctx, local_rank)   # all-reduces ordered on the context's stream
    else:
        ctx.set_phase_async(True)                # one share: nothing to combine, phases only enqueue
        comb = P.LocalCombiner([ctx], local_rank)
    stream = torch.cuda.ExternalStream(ctx.phase_stream(), device=torch.device("cuda", local_rank))
    for _ in range(args.warmup):
        P.step_shares([ctx], comb)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cross, dev_ms = 0, 0.0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        torch.cuda.synchronize(local_rank)
        e0.record(stream)   # the phases run on the context's stream
        st = P.step_shares([ctx], comb)[0]
        e1.record(stream)
        torch.cuda.synchronize(local_rank)
        dev_ms += e0.elapsed_time(e1)
        cross += st["crossings"]
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    if dist:
        t = torch.tensor([dev_ms, wall, float(cross)], dtype=torch.float64, device=f"cuda:{local_rank}")
        mx, sm = t.clone(), t.clone()
        tdist.all_reduce(mx, op=tdist.ReduceOp.MAX)
        tdist.all_reduce(sm, op=tdist.ReduceOp.SUM)
        dev_ms, wall, cross_all = float(mx[0]), float(mx[1]), float(sm[2])
    else:
        cross_all = float(cross)
    ctx.close()
    return {
        "metric": "ray-cell crossings/s", "value": cross_all / (dev_ms * 1e-3), "unit": "crossings/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded lognormal gas + L^-2 sources; the reference's inputs are not shipped)",
        "config": {"workload": _describe(spec), "timed_steps": f"{args.warmup + 1}..{args.warmup + args.steps}",
                   "graph": False, "l2": "state (>1 GB) larger than L2, no flush",
                   "parallelism": f"sources shared over {world} ranks, lit-cell rates all-reduced"},
        "e2e": {"value": cross_all / wall, "unit": "crossings/s",
                "h2d_bytes_per_step": 2 + 2 * len(W.grid_sources(inp)[1]), "d2h_bytes_per_step": 144 + 4},
        "gpu_launches": args.steps * launches_per_step(spec, args.ray_capacity),
        "clocks": clk,
        "crossings_per_step": cross_all / args.steps,
    }


def warm_up(ctx, args):
    """The W warm-up steps: graph steps, the last AUTOTUNE_STEPS of them taken by frt_autotune
    (real steps that also time candidate launch shapes; the chosen shapes are then captured in
    the step graph). Returns the chosen shapes, or None without autotuning."""
    n_tune = AUTOTUNE_STEPS if (not args.no_autotune and args.subgrid == "off"
                                and args.warmup >= AUTOTUNE_STEPS + 1) else 0
    for _ in range(args.warmup - n_tune):
        ctx.step(graph=not args.plain)
    if not n_tune:
        return None
    return ctx.autotune(n_tune)


def _tuning_config(t):
    if t is None:
        return "default shapes (no autotuning)"
    keys = ("raypass_block", "raypass_blocks_per_sm", "raypass_chunk", "walk_block", "walk_blocks_per_sm",
            "cellpass_blocks_per_sm", "split_blocks_per_sm", "steps")
    out = {k: int(t[k]) for k in keys}
    for k in ("raypass_blocks_per_sm", "cellpass_blocks_per_sm"):
        if out[k] == 0:
            out[k] = "resident (one wave)"
    out["measured_ns"] = {k: round(float(t[k]), 4) for k in ("raypass_ns_per_crossing", "walk_ns_per_ray",
                                                              "cellpass_ns_per_cell", "split_ns_per_ray")}
    return out


def run_ours(args, rank: int, world: int, local_rank: int):
    import numpy as np
    from flexrt_imaging_reion_b200 import workloads as W, rt
    spec = _spec(args.workload)
    inp = W.make_inputs(spec)
    ctx = rt.RTContext([inp], [args.seed + rank], precision="mixed", outputs="core",
                       ray_capacity=args.ray_capacity, lit_capacity=args.lit_capacity, device=local_rank)
    ctx.setup()
    if args.subgrid != "off":   # the sub-grid model on the synthetic RadHydro tables
        tables, consts = W.subgrid_inputs(spec.z)
        ctx.set_subgrid(tables, consts, ifront=(args.subgrid == "ifront"))
    ncell = spec.n ** 3
    itercount = ctx.itercount
    tuning = warm_up(ctx, args)
    dist = world > 1
    if dist:
        import torch
        import torch.distributed as tdist
        tdist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    cross = 0
    dev_ms = 0.0
    dark_ms = 0.0
    rp_ms = 0.0
    h2d = 2 * ctx.nbox + 2 * ctx.nsrc
    d2h = 0
    launches = 0
    lit = 0
    alive = moved = split = killed = 0
    per_step = launches_per_step(spec, args.ray_capacity, itercount)
    walk_ms, walked = 0.0, 0
    prev_alive = ctx.num_rays()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = ctx.step(graph=not args.plain)
        ms, dms = ctx.last_timing()
        cross += st["crossings"]
        dev_ms += ms
        dark_ms += dms
        rp_ms += ctx.last_raypass_ms()
        walk_ms += ctx.last_walk_ms()
        walked += prev_alive
        prev_alive = st["rays_alive"]
        launches += per_step
        lit += st["lit_cells"]
        alive += st["rays_alive"]
        moved += st["rays_moved"]
        split += st["rays_split"]
        killed += st["rays_killed"]
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    walk_bytes = WALK_BYTES_PER_RAY * walked + WALK_BYTES_PER_MOVED * moved + WALK_BYTES_PER_CROSSING * cross
    d2h = 144  # control block (per-step totals) read back each step
    # the state after the last timed step in the reference's restart formats: the CPU baseline
    # resumes the reference from it (a steady-state sample instead of the set-up-dominated first
    # steps)
    restart_files = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            restart_files = ctx.write_restart(0)
        except Exception:
            restart_files = None
    if dist:
        import torch
        import torch.distributed as tdist
        t = torch.tensor([dev_ms, wall, float(cross)], dtype=torch.float64, device=f"cuda:{local_rank}")
        mx = t.clone()
        tdist.all_reduce(mx, op=tdist.ReduceOp.MAX)
        sm = t.clone()
        tdist.all_reduce(sm, op=tdist.ReduceOp.SUM)
        dev_ms_max, wall_max, cross_all = float(mx[0]), float(mx[1]), float(sm[2])
    else:
        dev_ms_max, wall_max, cross_all = dev_ms, wall, float(cross)
    peak, peak_kind = _peaks()
    rp_gbs = RAYPASS_BYTES_PER_CROSSING * cross * itercount / (rp_ms * 1e-3) / 1e9 if rp_ms > 0 else None
    res = {
        "metric": "ray-cell crossings/s", "value": cross_all / (dev_ms_max * 1e-3), "unit": "crossings/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded lognormal gas + L^-2 sources; the reference's inputs are not shipped)",
        "config": {"workload": _describe(spec), "timed_steps": f"{args.warmup + 1}..{args.warmup + args.steps}",
                   "graph": not args.plain and args.subgrid != "ifront",
                   "subgrid": {"off": "none", "eq": "equilibrium sub-grid model (synthetic RadHydro tables)",
                               "ifront": "equilibrium sub-grid model with I-front tracking (synthetic RadHydro "
                                         "tables)"}[args.subgrid], "l2": "state (>1 GB) larger than L2, no flush",
                   "parallelism": "replicas" if world > 1 else "single",
                   "launch_shapes": _tuning_config(tuning)},
        "e2e": {"value": cross_all / wall_max, "unit": "crossings/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        # the dominant kernel: the ray pass (five launches per step, one per C2Ray iteration)
        "roofline": {"bound": "hbm", "kernel": "k_raypass_mixed (ray pass of one C2Ray iteration)",
                     "achieved": rp_gbs, "peak": peak, "unit": "GB/s",
                     "frac": (rp_gbs / peak) if rp_gbs else None,
                     "traffic": (RAYPASS_TRAFFIC_BYTES_PER_CROSSING * cross / args.steps
                                 if RAYPASS_TRAFFIC_BYTES_PER_CROSSING else None),
                     "traffic_note": "bytes per launch: ncu DRAM bytes per crossing of a ray pass x crossings per step",
                     "algorithmic_bytes_per_launch": RAYPASS_BYTES_PER_CROSSING * cross / args.steps,
                     "bytes_per_crossing": RAYPASS_BYTES_PER_CROSSING,
                     "peak_kind": peak_kind, "launch_ms": rp_ms / args.steps / itercount,
                     "launches_per_step": itercount},
        # the dark-cell pass runs on its own stream in the gaps of the lit-cell chain: its event
        # span is not its busy time, so it gets no roofline here (its serialised ncu time and
        # DRAM traffic are in the profiles)
        "dark_pass": {"kernel": "k_dark (cells no ray touched: whole step in one pass)",
                      "span_ms_per_step": dark_ms / args.steps, "bytes_per_cell": DARK_BYTES_PER_CELL,
                      "cells_per_step": ncell - lit / args.steps,
                      "traffic_per_step": DARK_TRAFFIC_BYTES_PER_CELL * (ncell - lit / args.steps),
                      "note": "CUDA-event span on its own stream, overlapped with the higher-priority "
                              "lit-cell chain; not its busy time"},
        # the walk: every live ray advanced, the moved rays' headers, segments and lit-cell marks
        # written
        "walk": {"kernel": "k_advance (update_rays: every live ray walked one step, the ray passes' "
                           "headers and packed segments written)",
                 "launch_ms": walk_ms / args.steps,
                 "algorithmic_bytes_per_launch": walk_bytes / args.steps,
                 "achieved": (walk_bytes / (walk_ms * 1e-3) / 1e9 if walk_ms > 0 else None),
                 "unit": "GB/s", "peak": peak,
                 "frac": (walk_bytes / (walk_ms * 1e-3) / 1e9 / peak if walk_ms > 0 and peak else None),
                 "rays_per_launch": walked / args.steps,
                 "bytes_per_ray": WALK_BYTES_PER_RAY, "bytes_per_moved_ray": WALK_BYTES_PER_MOVED,
                 "bytes_per_crossing": WALK_BYTES_PER_CROSSING},
        "gpu_launches": launches,
        "clocks": clk,
        "crossings_per_step": cross / args.steps,
        # each crossing is written once by the walk and read by each of the C2Ray iterations
        "segment_visits_per_step": cross * (1 + itercount) / args.steps,
        "lit_cells_per_step": lit / args.steps,
        "rays_alive_per_step": alive / args.steps,
        "rays_moved_per_step": moved / args.steps,
        "rays_split_per_step": split / args.steps,
        "rays_killed_per_step": killed / args.steps,
    }
    ctx.close()
    if restart_files is not None:
        res["_restart_files"] = restart_files
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # L runs 50 steps: 5 warm-up steps, then steps 6..50 timed
    ap.add_argument("--steps", type=int, default=45)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["L", "M", "S", "E", "A"], default="L")
    ap.add_argument("--no-loop", action="store_true", help="E: skip the per-box launch-loop comparison")
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--ray-capacity", type=int, default=16 << 20)
    ap.add_argument("--lit-capacity", type=int, default=0, help="0 = all cells")
    ap.add_argument("--plain", action="store_true", help="launch kernels directly instead of the CUDA graph")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--cpu-baseline-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # the reference arm times the same step window as this arm (about 8-10 s per L step on 16 cores)
    ap.add_argument("--ref-time-cap", type=float, default=900.0)
    ap.add_argument("--subgrid", choices=["off", "eq", "ifront"], default="off",
                    help="single boxes: run the sub-grid model (eq) or the sub-grid model with I-front tracking "
                         "(ifront) on synthetic RadHydro tables; no CPU baseline or reference arm for these")
    ap.add_argument("--mode", choices=["replicas", "partition"], default="replicas",
                    help="N>1 on one box: N independent replicas (weak), or the box's sources shared "
                         "over the N ranks with the lit cells' rates all-reduced (strong)")
    args = ap.parse_args()
    if args.subgrid != "off":
        args.no_cpu_baseline = True   # the reference arm and the CPU baseline time the plain model
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return
        if args.workload == "E":
            try:
                cr, wt, nb = run_reference_ensemble(args.warmup + args.steps, threads, args.ref_time_cap, args.seed)
            except Exception as e:
                print(json.dumps({"impl": "reference", "unavailable": f"compiled reference failed: {e}"}))
                return
            v = cr / wt if wt > 0 else None
            from flexrt_imaging_reion_b200 import workloads as W
            print(json.dumps({
                "impl": "reference", "metric": "ray-cell crossings/s", "value": v, "unit": "crossings/s",
                "n_gpus": world, "steps": args.warmup + args.steps, "warmup": 0,
                "ms_per_step": None, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f32+f64 (reference float storage, double locals)", "data": "synthetic",
                "config": {"workload": _describe_ensemble(W.config_E())},
                "cpu_baseline": {"value": v, "unit": "crossings/s", "cores": threads, "kind": "reference",
                                 "sample": f"first {nb} boxes of the ensemble, {args.warmup + args.steps} steps each, "
                                           f"OpenMP {threads} threads (time cap {args.ref_time_cap:.0f} s)"},
                "e2e": {"value": v, "unit": "crossings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            }))
            return
        spec = _spec(args.workload)
        try:
            rows, setup = run_reference(spec, args.workload, args.warmup + args.steps, threads, args.ref_time_cap,
                                        args.seed)
        except Exception as e:  # the reference arm must print a line even when it cannot run
            print(json.dumps({"impl": "reference", "unavailable": f"compiled reference failed: {e}"}))
            return
        timed = rows[args.warmup:] if len(rows) > args.warmup else rows
        cr = sum(c for c, _ in timed)
        wt = sum(w for _, w in timed)
        v = cr / wt if wt > 0 else None
        print(json.dumps({
            "impl": "reference", "metric": "ray-cell crossings/s", "value": v, "unit": "crossings/s",
            "n_gpus": world, "steps": len(timed), "warmup": min(args.warmup, len(rows)),
            "ms_per_step": 1e3 * wt / max(1, len(timed)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64 (reference float storage, double locals)", "data": "synthetic",
            "config": {"workload": _describe(spec), "timed_steps": f"{min(args.warmup, len(rows)) + 1}.."
                       f"{len(rows)}", "setup_s": setup},
            "cpu_baseline": {"value": v, "unit": "crossings/s", "cores": threads, "kind": "reference",
                             "sample": f"{len(timed)} timed steps after {min(args.warmup, len(rows))} warm-up steps, "
                                       f"OpenMP {threads} threads (time cap {args.ref_time_cap:.0f} s)"},
            "e2e": {"value": v, "unit": "crossings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=120))
    if args.workload == "A":
        if rank == 0:
            print(json.dumps(run_adjoint(args)))
        return
    if args.workload == "E":
        res = run_ensemble(args, rank, world, local_rank)
    elif args.mode == "partition":
        res = run_partition(args, rank, world, local_rank)
    else:
        res = run_ours(args, rank, world, local_rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "E":
        try:
            cr, wt, nb = run_reference_ensemble(args.cpu_baseline_steps, threads, 30.0, args.seed)
            res["cpu_baseline"] = {"value": cr / wt if wt else None, "unit": "crossings/s", "cores": threads,
                                   "kind": "reference",
                                   "sample": f"steps 1..{args.cpu_baseline_steps} of the first {nb} boxes, reference "
                                             f"OpenMP code compiled from its sources (one build per grid size)"}
        except Exception as e:
            res["cpu_baseline"] = {"value": None, "unit": "crossings/s", "cores": threads, "kind": "reference",
                                   "sample": f"unavailable: {e}"}
    restart_files = res.pop("_restart_files", None)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload != "E":
        spec = _spec(args.workload)
        last = args.warmup + args.steps
        try:
            if restart_files is None:
                raise RuntimeError("no restart records of the device state")
            rows, setup = run_reference_restart(spec, args.workload + "_restart", restart_files,
                                                args.cpu_baseline_steps, threads, args.seed)
            sample = (f"steps {last + 1}..{last + len(rows)} of the same workload: the device state after step "
                      f"{last} written in the reference's restart formats and resumed by the reference's own "
                      f"restart path (input_grid = TRUE; restart set-up and the reference's balance_cpus over the restored "
                      f"rays, {setup:.1f} s, excluded); reference "
                      f"OpenMP code compiled from its sources, {threads} threads")
        except Exception as e:
            # no restart build: the first steps from a fresh start (set-up-dominated, labelled so)
            rows, setup = run_reference(spec, args.workload, args.cpu_baseline_steps, threads, 60.0, args.seed)
            sample = (f"steps 1..{len(rows)} of the same workload from a fresh start (set-up {setup:.1f} s "
                      f"excluded; the restart sample was unavailable: {e}), reference OpenMP code compiled "
                      f"from its sources, {threads} threads")
        try:
            cr = sum(r[0] for r in rows)
            wt = sum(r[1] for r in rows)
            res["cpu_baseline"] = {"value": cr / wt if wt else None, "unit": "crossings/s", "cores": threads,
                                   "kind": "reference", "sample": sample}
            if rows and len(rows[0]) > 2:
                res["cpu_baseline"]["per_step"] = [r[2] for r in rows]
        except Exception as e:
            res["cpu_baseline"] = {"value": None, "unit": "crossings/s", "cores": threads, "kind": "reference",
                                   "sample": f"unavailable: {e}"}
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()
    if rank == 0:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
