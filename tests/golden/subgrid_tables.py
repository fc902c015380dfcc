"""Synthetic sub-grid tables in the reference's own file formats (test infrastructure).

The reference's sub-grid model reads RadHydro tables that are not shipped with it:

* 27 files (3 photo-ionisation rates x 3 reionisation redshifts x 3 overdensities), each Nt = 5000
  rows of 5 numbers -- time since ionisation [yr], the frequency-averaged and the 912 A mean free
  paths [comoving Mpc/h], the HI fraction and the temperature [K] (import_subgrid_file,
  subgrid.cc:20-47; names and folder subgrid.cc:151-173, "equilibrium/" with suffix "_noclump");
* delta_over_sigma_table.txt: a line of n_dlin = 500 cosmic times [s], a line of 500 values of
  linear overdensity / sigma, then 500 lines of 500 non-linear overdensities, one line per time
  (import_delta_over_sigma_table, subgrid.cc:49-95).

Here they are the smooth closed-form functions of flexrt_imaging_reion_b200.workloads (the
package's synthetic inputs), written with 17 significant digits so that the reference's
fscanf("%le") and the in-memory arrays give the same doubles (and the same floats after the
reference's (float) casts). The same arrays feed the oracle and the device; nothing here is
taken from the RadHydro simulations, which are not available.
"""
from __future__ import annotations

import os
from typing import Dict

import numpy as np

from flexrt_imaging_reion_b200 import workloads as W

NT = W.SG_NT
N_DLIN = W.SG_NDLIN
GAMMA_TAGS = ["G14", "G13", "G12"]
ZRE_TAGS = ["zre12", "zre8", "zre6"]
DENSITY_TAGS = ["dm3", "d0", "dp3"]


def radhydro() -> Dict[str, np.ndarray]:
    """Per file (q gamma, m zre, p density, in the reference's loop order) the 5 columns."""
    return W.subgrid_radhydro()


def table_span(cosmic_time_s):
    """The cosmic times [s] the overdensity table spans: z = 16 to z = 4.5."""
    return cosmic_time_s(1.0 / 17.0), cosmic_time_s(1.0 / 5.5)


def delta_over_sigma(t0: float, t1: float) -> Dict[str, np.ndarray]:
    """The linear -> non-linear overdensity table (flexrt_imaging_reion_b200.workloads)."""
    return W.subgrid_delta_over_sigma(t0, t1)


def write_reference_files(directory: str, cosmic_time_s) -> None:
    """The tables in the folder layout the reference reads them from (subgrid_dir = directory)."""
    rh = radhydro()
    eq = os.path.join(directory, "equilibrium")
    os.makedirs(eq, exist_ok=True)
    for q in range(3):
        for m in range(3):
            for p in range(3):
                name = f"{GAMMA_TAGS[q]}_{ZRE_TAGS[m]}_{DENSITY_TAGS[p]}_noclump.txt"
                c = rh["cols"][q, m, p]
                with open(os.path.join(eq, name), "w") as f:
                    for k in range(NT):
                        f.write("%.17e %.17e %.17e %.17e %.17e\n" % (rh["time_yr"][k], c[0, k], c[1, k], c[2, k],
                                                                      c[3, k]))
    ds = delta_over_sigma(*table_span(cosmic_time_s))
    with open(os.path.join(directory, "delta_over_sigma_table.txt"), "w") as f:
        f.write(" ".join("%.17e" % v for v in ds["t"]) + "\n")
        f.write(" ".join("%.17e" % v for v in ds["ds"]) + "\n")
        for i in range(N_DLIN):
            f.write(" ".join("%.17e" % v for v in ds["dnl"][i]) + "\n")


def cosmic_time_from_table(path: str):
    """cosmic_time(a) of the reference (cosmo_funcs.cc:42-49) over its binary table of 100000
    (a, t) double pairs, in double (the table's own precision) and then rounded to float."""
    raw = np.fromfile(path, dtype=np.float64).reshape(-1, 2)
    a_tab, t_tab = raw[:, 0], raw[:, 1]
    n = len(a_tab)

    def ct(a: float) -> float:
        a = float(np.float32(a))
        ind = int(np.floor((a - a_tab[0]) / (a_tab[n - 1] - a_tab[0]) * (n - 1)))
        return float(np.float32(t_tab[ind] + (t_tab[ind + 1] - t_tab[ind]) / (a_tab[ind + 1] - a_tab[ind]) *
                                (a - a_tab[ind])))
    return ct


def reference_arrays(t0: float, t1: float) -> Dict[str, np.ndarray]:
    """The tables as the reference holds them in memory after reading the files: time_RH and
    fh1_RH as flat [Nt][3][3][3] floats written at the gamma index q + 1 (gam_offset,
    subgrid.cc:24-36), with one slot more for the last row's spill; times in s (time_RH *= yr_to_s,
    float); the overdensity table as floats."""
    return W.subgrid_arrays(t0, t1)
