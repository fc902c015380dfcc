"""Parity helpers: run the CUDA path and the CPU oracle on the same seeded box and compare.

Tolerances (stated per quantity, checked per cell / per ray):
  * ray tree: (cell, order, pixel, itheta) exact; geometry (x, y, z, r, dr, direction) bit-exact
    except for rays that went through a merge (photon-weighted float sums: 1e-5 relative);
  * ray photon counts: 1e-4 relative (mixed precision) / 1e-6 (strict);
  * Gamma_HI, Gamma_HeI per cell: 1e-4 relative where the oracle value is above 1e-6 of the box
    maximum (mixed) / 1e-6 (strict), and both zero where the oracle has no deposit;
  * x_HI (f_H1) and avg x_HI: 1e-4 absolute; T: 1e-4 relative.
A ray whose photon count sits within 1e-4 of the removal threshold nphot_min (or of a split
threshold) may legitimately be kept by one side and removed by the other; such near-tie rays are
reported separately and not counted as mismatches.
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


def oracle_states(inp: W.BoxInputs, seed: int, steps: int) -> List[Dict[str, np.ndarray]]:
    """States of the CPU oracle after the set-up (index 0) and after each step."""
    o = O.Oracle(inp, seed)
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


DEVICE_FIELDS = {
    "nH": "NH", "nHe": "NHE", "nH1": "NH1", "nHe1": "NHE1", "ne": "NE", "f_H1": "F_H1", "f_He1": "F_HE1",
    "f_H2": "F_H2", "temp": "TEMP", "avg_nh1": "AVG_NH1", "avg_nhe1": "AVG_NHE1", "gamma_H1_tot": "GAMMA_H1_TOT",
    "gamma_He1_tot": "GAMMA_HE1_TOT", "heat_rate": "HEAT_RATE", "cool_rate": "COOL_RATE", "treion": "TREION",
    "gamma_H1_nu": "GAMMA_H1_NU", "gamma_He1_nu": "GAMMA_HE1_NU", "ngam_nu": "NGAM_NU", "rho": "RHO",
}
DIAG_FIELDS = {"mfp": "MFP", "mfp_912": "MFP_912", "recrate_H2": "RECRATE_H2", "n_tot": "N_TOT",
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
    for k in ("gamma_H1_tot", "gamma_He1_tot"):
        a, b = dev[k], ref[k]
        floor = max(float(np.abs(b).max()) * 1e-6, 1e-300)
        r = _rel(a, b, floor)
        out[k + "_maxrel"] = float(r.max()) if r.size else 0.0
        out[k + "_bad"] = int((r > rel_gamma).sum())
        out[k + "_zero_mismatch"] = int(((a == 0) != (b == 0)).sum())
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


def compare_rays(dev: Dict[str, np.ndarray], ref: Dict[str, np.ndarray], nphot_min: float, rel_nphot: float,
                 exact_geom: bool = True) -> Dict[str, float]:
    """Multiset comparison of the live rays (pool order differs from the reference's slot order)."""
    kd = _ray_keys(dev, exact_geom)
    kr = _ray_keys(ref, exact_geom)
    from collections import defaultdict
    idx = defaultdict(list)
    for i, k in enumerate(kr):
        idx[k].append(i)
    matched_d, matched_r = [], []
    unmatched_d = []
    for i, k in enumerate(kd):
        lst = idx.get(k)
        if lst:
            matched_r.append(lst.pop())
            matched_d.append(i)
        else:
            unmatched_d.append(i)
    unmatched_r = [i for lst in idx.values() for i in lst]
    md, mr = np.array(matched_d, int), np.array(matched_r, int)
    out = {"n_dev": len(kd), "n_ref": len(kr), "matched": len(md)}
    if len(md):
        gd, gr = dev["ray_geom"][md], ref["ray_geom"][mr]
        out["geom_exact"] = bool((gd.view(np.uint32) == gr.view(np.uint32)).all())
        out["geom_maxrel"] = float(_rel(gd, gr, 1e-30).max())
        npd, npr = dev["ray_nphot"][md], ref["ray_nphot"][mr]
        floor = max(float(np.abs(npr).max()) * 1e-7, 1e-300)
        r = _rel(npd, npr, floor)
        out["nphot_maxrel"] = float(r.max())
        out["nphot_bad"] = int((r.max(axis=1) > rel_nphot).sum())
    else:
        out.update(geom_exact=True, geom_maxrel=0.0, nphot_maxrel=0.0, nphot_bad=0)

    def near_tie(st, ids):
        s = st["ray_nphot"][ids].astype(np.float64).sum(axis=1) if len(ids) else np.zeros(0)
        return int((np.abs(s / nphot_min - 1.0) < 1e-3).sum()) if nphot_min > 0 else 0

    out["unmatched_dev"] = len(unmatched_d)
    out["unmatched_ref"] = len(unmatched_r)
    out["unmatched_near_tie"] = near_tie(dev, unmatched_d) + near_tie(ref, unmatched_r)
    return out
