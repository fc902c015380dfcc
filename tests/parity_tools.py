"""Parity helpers: run the CUDA path and the CPU oracle on the same seeded box and compare.

Tolerances (stated per quantity, checked per cell / per ray):
  * ray tree: (cell, order, pixel, itheta) exact; geometry (x, y, z, r, dr, direction) bit-exact
    except for rays that went through a merge (photon-weighted float sums: 1e-5 relative);
  * ray photon counts: 1e-4 relative (mixed precision) / 1e-6 (strict);
  * Gamma_HI, Gamma_HeI per cell: 1e-4 relative (mixed) / 1e-5 (strict) in every cell, plus an
    absolute allowance of GAMMA_SUBNORMAL = 128 FLT_MIN (1.5e-36 s^-1) for the float subnormal
    range, and zero exactly where the oracle has no deposit above that allowance. The device sums
    a cell's deposits with float atomics (PTX atom / red .add.f32), which flush subnormal inputs
    and results to zero, while the reference's CPU sums keep them; and a sum that is itself
    subnormal carries an absolute, not relative, precision of 2^-149. Rates below 1e-36 s^-1 are
    24 orders of magnitude below those of ionised gas and change no ionised fraction. A cell whose
    rate is made of the last photons of rays at the removal threshold (a ray whose photon total
    falls below nphot_min deposits all of it and stops, ray_tracing.cc:782-812) may further differ
    by at most the rate one such ray gives it, nphot_min / (dt V <n>): those cells are counted
    apart and bounded (THRESHOLD_CELLS);
  * x_HI (f_H1) and avg x_HI: 1e-4 absolute; T: 1e-3 relative (mixed) / 1e-4 (strict);
  * photon ledger of a step (emitted, deposited, killed, in flight) against the oracle's own
    ledger: 1e-6 of the photons emitted since the start.
A ray whose photon count sits within 1e-4 (relative) of the removal threshold nphot_min may
legitimately be kept by one side and removed by the other (the ray photon counts themselves are
held to 1e-4); such near-tie rays are reported separately, and the tests bound their number.
"""
from __future__ import annotations

import os
import sys
import tempfile
from typing import Dict, List

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)

from oracle import frtd  # noqa: E402
from oracle import oracle as O  # noqa: E402
from flexrt_imaging_reion_b200 import workloads as W  # noqa: E402

# relative distance of a ray's photon count from nphot_min within which keep / remove may differ
NEAR_TIE = 1e-4
# absolute allowance on a cell's Gamma for the float subnormal range: 128 x FLT_MIN = 2^-119
GAMMA_SUBNORMAL = 128.0 * float(np.finfo(np.float32).tiny)
PHOT_NORM = 1e60   # the photon-count normalisation of the ray records (phot_norm)


def threshold_cells_bound(ncell: int) -> int:
    """Most cells of a box whose rate may differ by up to one threshold ray's rate."""
    return 2 + ncell // 10000


def oracle_states(inp: W.BoxInputs, seed: int, steps: int, tau_max: float = 0.0) -> List[Dict[str, np.ndarray]]:
    """States of the CPU oracle after the set-up (index 0) and after each step (with the opt-in
    optical-depth limit tau_max when it is > 0)."""
    o = O.Oracle(inp, seed)
    if tau_max > 0:
        o.set_tau_limit(tau_max)
    out = []
    with tempfile.TemporaryDirectory() as td:
        for s in range(steps + 1):
            if s > 0:
                o.step()
            p = os.path.join(td, f"s{s}.frtd")
            o.dump(p)
            out.append(frtd.read(p))
    o.close()
    return out


def oracle_iter(inp: W.BoxInputs, seed: int, steps: int):
    """The same states as oracle_states, one at a time (for boxes whose states are too large to
    hold all at once)."""
    o = O.Oracle(inp, seed)
    try:
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, "s.frtd")
            for s in range(steps + 1):
                if s > 0:
                    o.step()
                o.dump(p)
                yield frtd.read(p)
    finally:
        o.close()


DEVICE_FIELDS = {
    "nH": "NH", "nHe": "NHE", "nH1": "NH1", "nHe1": "NHE1", "ne": "NE", "f_H1": "F_H1", "f_He1": "F_HE1",
    "f_H2": "F_H2", "temp": "TEMP", "avg_nh1": "AVG_NH1", "avg_nhe1": "AVG_NHE1", "gamma_H1_tot": "GAMMA_H1_TOT",
    "gamma_He1_tot": "GAMMA_HE1_TOT", "heat_rate": "HEAT_RATE", "cool_rate": "COOL_RATE", "treion": "TREION",
    "rho": "RHO",
}
# per-bin rates and photon counts are kept by the device only with diag outputs (or strict precision)
DIAG_FIELDS = {"gamma_H1_nu": "GAMMA_H1_NU", "gamma_He1_nu": "GAMMA_HE1_NU", "ngam_nu": "NGAM_NU", "mfp": "MFP", "mfp_912": "MFP_912", "recrate_H2": "RECRATE_H2", "n_tot": "N_TOT",
               "dne_dt": "DNE_DT", "IF_speed": "IF_SPEED", "u_nu": "U_NU"}


def device_state(ctx, box: int = 0, diag: bool = False) -> Dict[str, np.ndarray]:
    st = {}
    names = dict(DEVICE_FIELDS)
    if diag:
        names.update(DIAG_FIELDS)
    for k, f in names.items():
        st[k] = ctx.get_field(box, f)
    st["treion_flag"] = ctx.get_field(box, "TREION_FLAG").astype(np.uint8)
    st.update(ctx.rays(box))
    return st


def _rel(a: np.ndarray, b: np.ndarray, floor: float) -> np.ndarray:
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    den = np.maximum(np.abs(b), floor)
    return np.abs(a - b) / den


def compare_fields(dev: Dict[str, np.ndarray], ref: Dict[str, np.ndarray], rel_gamma: float, abs_x: float,
                   rel_t: float) -> Dict[str, float]:
    """Worst-case errors of the headline fields; keys ending in _bad count violating cells."""
    out = {}
    sc = ref["scalars"]
    nphot_min, dt, dx = float(sc[2]), float(sc[1]), float(sc[8])
    for k, avg in (("gamma_H1_tot", "avg_nh1"), ("gamma_He1_tot", "avg_nhe1")):
        a, b = dev[k].astype(np.float64), ref[k].astype(np.float64)
        diff = np.abs(a - b)
        normal = np.abs(b) > GAMMA_SUBNORMAL
        # relative per cell wherever the oracle's rate is above the subnormal allowance
        r = diff[normal] / np.abs(b[normal])
        out[k + "_maxrel"] = float(r.max()) if r.size else 0.0
        within = diff <= rel_gamma * np.abs(b) + GAMMA_SUBNORMAL
        # the rate one ray at the removal threshold gives the cell (all its photons absorbed)
        with np.errstate(divide="ignore"):
            g_thr = nphot_min * PHOT_NORM / dt / dx ** 3 / np.maximum(ref[avg].astype(np.float64), 1e-300)
        thr = ~within & (diff <= g_thr)
        out[k + "_threshold_cells"] = int(thr.sum())
        out[k + "_bad"] = int((~within & ~thr).sum())
        out[k + "_zero_mismatch"] = int((((a == 0) != (b == 0)) & (np.maximum(np.abs(a), np.abs(b)) > GAMMA_SUBNORMAL)).sum())
        # cells with a rate on either side inside the allowance (reported, not failed)
        out[k + "_subnormal_cells"] = int((((a != 0) | (b != 0)) & (np.maximum(np.abs(a), np.abs(b)) <= GAMMA_SUBNORMAL)).sum())
    for k in ("f_H1", "f_He1"):
        d = np.abs(dev[k].astype(np.float64) - ref[k].astype(np.float64))
        out[k + "_maxabs"] = float(d.max())
        out[k + "_bad"] = int((d > abs_x).sum())
    for k in ("avg_nh1",):
        d = np.abs(dev[k].astype(np.float64) - ref[k].astype(np.float64)) / ref["nH"].astype(np.float64)
        out["avg_xHI_maxabs"] = float(d.max())
        out["avg_xHI_bad"] = int((d > abs_x).sum())
    r = _rel(dev["temp"], ref["temp"], 1.0)
    out["temp_maxrel"] = float(r.max())
    out["temp_bad"] = int((r > rel_t).sum())
    out["treion_flag_mismatch"] = int((dev["treion_flag"] != ref["treion_flag"]).sum())
    return out


def _ray_keys(st: Dict[str, np.ndarray], exact_geom: bool):
    g = st["ray_geom"]
    keys = []
    for i in range(len(st["ray_order"])):
        k = (int(st["ray_cell"][i]), int(st["ray_order"][i]), int(st["ray_pixel"][i]), int(st["ray_itheta"][i]))
        if exact_geom:
            k = k + tuple(g[i, [5, 6, 7, 3]].view(np.uint32).tolist())
        keys.append(k)
    return keys


def _match(kd, kr, cand_d, cand_r, fd=None, fr=None):
    """Pair rays with equal keys. Several rays can share a key (same cell, order, pixel and
    angle index, e.g. two merged rays of one bin in consecutive steps); with feature vectors
    fd / fr (photon count and position) the rays of such a key group are paired by the
    permutation with the least feature distance (greedy for groups above six rays)."""
    import itertools
    from collections import defaultdict
    idx_r, idx_d = defaultdict(list), defaultdict(list)
    for i in cand_r:
        idx_r[kr[i]].append(i)
    for i in cand_d:
        idx_d[kd[i]].append(i)
    md, mr, ud, ur = [], [], [], []
    for k, ld in idx_d.items():
        lr = idx_r.pop(k, [])
        if fd is not None and len(ld) > 1 and len(lr) > 1:
            n = min(len(ld), len(lr))
            cost = lambda i, j: float(np.abs(fd[i] - fr[j]).sum())
            if max(len(ld), len(lr)) <= 6:
                best = None
                for perm in itertools.permutations(range(len(lr)), n):
                    c = sum(cost(ld[q], lr[perm[q]]) for q in range(n))
                    if best is None or c < best[0]:
                        best = (c, perm)
                pd = ld[:n]
                pr = [lr[q] for q in best[1]]
            else:
                pd, pr, free = [], [], list(lr)
                for i in ld[:n]:
                    j = min(free, key=lambda j: cost(i, j))
                    free.remove(j)
                    pd.append(i)
                    pr.append(j)
            md += pd
            mr += pr
            ud += [i for i in ld if i not in pd]
            ur += [j for j in lr if j not in pr]
            continue
        n = min(len(ld), len(lr))
        md += ld[:n]
        mr += lr[:n]
        ud += ld[n:]
        ur += lr[n:]
    for lr in idx_r.values():
        ur += lr
    return md, mr, ud, ur


def _features(st: Dict[str, np.ndarray], dx: float) -> np.ndarray:
    """log photon count and position in cells, for pairing rays that share a key."""
    if not len(st["ray_order"]):
        return np.zeros((0, 4))
    s = np.log(np.maximum(st["ray_nphot"].astype(np.float64).sum(axis=1), 1e-300))
    pos = st["ray_geom"][:, 5:8].astype(np.float64) / dx
    return np.concatenate([s[:, None], pos], axis=1)


def compare_rays(dev: Dict[str, np.ndarray], ref: Dict[str, np.ndarray], nphot_min: float, rel_nphot: float,
                 rel_geom_merged: float = 1e-5, dx: float = 1.0, dx0: float = 1.0,
                 rel_nphot_merged: float = 1e-3) -> Dict[str, float]:
    """Multiset comparison of the live rays (pool order differs from the reference's slot order).

    Pass 1 matches rays on (cell, order, pixel, itheta) plus the exact bits of x, y, z, r (every
    ray that was only advanced / split / cast). Pass 2 matches the remaining rays on the integer
    key alone and checks their geometry (rays whose x, y, z, r, dr are photon-weighted float sums
    of a merge) to rel_geom_merged of the cell size: r, dr against dx0 (comoving), x, y, z against dx."""
    kd, kr = _ray_keys(dev, True), _ray_keys(ref, True)
    md, mr, ud, ur = _match(kd, kr, range(len(kd)), range(len(kr)))
    kd2, kr2 = _ray_keys(dev, False), _ray_keys(ref, False)
    md2, mr2, ud2, ur2 = _match(kd2, kr2, ud, ur, _features(dev, dx), _features(ref, dx))
    out = {"n_dev": len(kd), "n_ref": len(kr), "matched_exact": len(md), "matched_merged": len(md2)}
    out["geom_exact"] = True
    if md2:
        gd, gr = dev["ray_geom"][md2].astype(np.float64), ref["ray_geom"][mr2].astype(np.float64)
        scale = np.array([dx0, dx0, dx, dx, dx])
        r = np.abs(gd[:, 3:8] - gr[:, 3:8]) / scale
        out["merged_geom_maxrel"] = float(r.max())
        out["merged_geom_bad"] = int((r.max(axis=1) > rel_geom_merged).sum())
    else:
        out["merged_geom_maxrel"] = 0.0
        out["merged_geom_bad"] = 0
    # photon counts: rays matched exactly to rel_nphot; merged rays (float sums over the rays of a
    # bin, accumulated in another order) to rel_nphot_merged
    out.update(nphot_maxrel=0.0, nphot_bad=0, nphot_merged_maxrel=0.0, nphot_merged_bad=0, dir_maxabs=0.0)
    allref = ref["ray_nphot"]
    floor = max(float(np.abs(allref).max()) * 1e-7, 1e-300) if allref.size else 1e-300
    for lab, ids_d, ids_r, tol in (("", md, mr, rel_nphot), ("_merged", md2, mr2, rel_nphot_merged)):
        if not ids_d:
            continue
        # per-bin differences relative to the ray's photon total: a strongly attenuated bin
        # (tau ~ 10 along the ray) turns a 1e-6 change of the gathered densities into a 1e-5
        # change of its own, negligible, photon count
        nd = dev["ray_nphot"][ids_d].astype(np.float64)
        nr = ref["ray_nphot"][ids_r].astype(np.float64)
        den = np.maximum(np.abs(nr).sum(axis=1, keepdims=True), floor)
        r = np.abs(nd - nr) / den
        out[f"nphot{lab}_maxrel"] = float(r.max())
        bad = np.nonzero(r.max(axis=1) > tol)[0]
        out[f"nphot{lab}_bad"] = int(len(bad))
        # the first few offenders: key, photon sums and radii on both sides
        out[f"nphot{lab}_worst"] = [
            (kd2[ids_d[j]], float(dev["ray_nphot"][ids_d[j]].sum()), float(ref["ray_nphot"][ids_r[j]].sum()),
             float(dev["ray_geom"][ids_d[j], 3]), float(ref["ray_geom"][ids_r[j], 3])) for j in bad[:3]]
    ma, mb = np.array(md + md2, int), np.array(mr + mr2, int)
    if len(ma):
        hd, hr = dev["ray_geom"][ma, 0:3], ref["ray_geom"][mb, 0:3]
        out["dir_maxabs"] = float(np.abs(hd.astype(np.float64) - hr).max())

    # the optical-depth limit (opt-in, oracle dumps with "ray_col"): the columns of the matched
    # rays, and rays whose optical depth ties with the limit count as near ties
    tau = None
    if "ray_col" in ref and "ray_col" in dev and "tau_sigma" in ref:
        tau = (float(ref["tau_max"][0]), ref["tau_sigma"].astype(np.float64))
        out["col_maxrel"] = 0.0
        if len(ma):
            cd, cr = dev["ray_col"][ma].astype(np.float64), ref["ray_col"][mb].astype(np.float64)
            den = np.maximum(np.abs(cr), 1.0)
            out["col_maxrel"] = float((np.abs(cd - cr) / den).max())

    def near_tie(st, ids):
        s = st["ray_nphot"][ids].astype(np.float64).sum(axis=1) if len(ids) else np.zeros(0)
        tie = (np.abs(s / nphot_min - 1.0) < NEAR_TIE) if nphot_min > 0 else np.zeros(len(s), bool)
        if tau is not None and len(ids):
            tmax, sig = tau
            col = st["ray_col"][ids].astype(np.float64)
            tmin = (col[:, :1] * sig[0][None, :] + col[:, 1:2] * sig[1][None, :]).min(axis=1)
            tie |= np.abs(tmin / tmax - 1.0) < NEAR_TIE
        return int(tie.sum())

    out["unmatched_dev"] = len(ud2)
    out["unmatched_ref"] = len(ur2)
    out["unmatched_near_tie"] = near_tie(dev, ud2) + near_tie(ref, ur2)
    return out


def compare_ledger(stats: Dict[str, float], ref: Dict[str, np.ndarray], emitted_total: float) -> Dict[str, float]:
    """Device photon totals of one step against the oracle's ledger of the same step (emitted,
    deposited on the last C2Ray iteration, killed, dumped-and-killed overlap, in flight after the
    step), each difference divided by the photons emitted since the start of the run."""
    led = ref["ledger"]
    keys = ("photons_emitted", "photons_deposited", "photons_killed", "photons_overlap", "photons_in_flight")
    return {k: abs(float(stats[k]) - float(led[j])) / emitted_total for j, k in enumerate(keys)}


def photon_budget(stats_list, in_flight_0: float) -> float:
    """Relative closure of the photon ledger over the steps: in-flight(start) + emitted - (deposited -
    overlap) - killed - in-flight(end), divided by the photons emitted (set-up cast included)."""
    emitted = in_flight_0
    dep = kil = ovl = 0.0
    for st in stats_list:
        emitted += st["photons_emitted"]
        dep += st["photons_deposited"]
        kil += st["photons_killed"]
        ovl += st["photons_overlap"]
    end = stats_list[-1]["photons_in_flight"]
    return abs(emitted - (dep - ovl) - kil - end) / emitted


def oracle_restart_states(inp: W.BoxInputs, seed: int, files, steps: int) -> List[Dict[str, np.ndarray]]:
    """States of the oracle restarted from (gas, treion, rays) records, after the read (index 0)
    and after each step."""
    o = O.Oracle(inp, seed)
    o.read_restart(*files)
    out = []
    with tempfile.TemporaryDirectory() as td:
        for s in range(steps + 1):
            if s > 0:
                o.step()
            p = os.path.join(td, f"s{s}.frtd")
            o.dump(p)
            out.append(frtd.read(p))
    o.close()
    return out
