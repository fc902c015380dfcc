"""ORACLE TEST INFRASTRUCTURE -- not part of the product.

ctypes front end of the CPU restatement in oracle/frt_oracle.cc, plus the build recipe for it.
Only the tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, and only
as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")

sys.path.insert(0, REPO)
from flexrt_imaging_reion_b200 import workloads as W  # noqa: E402

# The alpha = 1.5 interpolation of the reference's 5-bin spectrum table (set_spectrum,
# gas_funcs.cc:44-70) lands on index floor(2/3.5*14) = 8, i.e. it interpolates between the rows
# alpha = 1.5 and 1.75 at weight 0 (input_files/spectrum_tables_5bins.txt lines 10-11). Only the
# alpha column and those two rows enter the arithmetic.
SPEC_ALPHA = [-0.5 + 0.25 * i for i in range(15)]
SPEC_ROWS = {8: [0.2, 0.2, 0.2, 0.2, 0.2], 9: [0.221, 0.213, 0.203, 0.191, 0.172]}


class Params(C.Structure):
    _fields_ = [("N", C.c_int), ("F", C.c_int), ("path_length", C.c_int), ("itercount", C.c_int),
                ("ray_per_cell_max", C.c_int), ("hpx_lvl", C.c_int), ("nu_eV", C.c_double * 8),
                ("spectrum_alpha", C.c_double * 15), ("spectrum_table", (C.c_double * 8) * 15),
                ("cl_factor", C.c_float), ("box_hmpc", C.c_float), ("z", C.c_float), ("const_clump", C.c_float),
                ("rkill_cm", C.c_double), ("seed", C.c_uint)]


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "frt_oracle.cc")
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(REPO, "flexrt_imaging_reion_b200", "csrc",
                                                                 "hp_nest.h"))):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=gnu++17", "-ffp-contract=off", "-fPIC", "-shared", "-w", "-I", HERE,
                    src, "-o", LIB], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.orc_create.restype = C.c_void_p
        _lib.orc_create.argtypes = [C.POINTER(Params), C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_step.argtypes = [C.c_void_p]
        _lib.orc_num_rays.restype = C.c_long
        _lib.orc_num_rays.argtypes = [C.c_void_p]
        _lib.orc_last_crossings.restype = C.c_long
        _lib.orc_last_crossings.argtypes = [C.c_void_p]
        _lib.orc_dump.argtypes = [C.c_void_p, C.c_char_p]
        _lib.orc_scalars.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_destroy.argtypes = [C.c_void_p]
        _lib.orc_rotate.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        _lib.orc_pix2vec.argtypes = [C.c_int, C.c_int, C.c_void_p]
        _lib.orc_vec2pix.argtypes = [C.c_int, C.c_void_p]
        _lib.orc_vec2pix.restype = C.c_int
        for fn in ("orc_write_gas", "orc_write_rays", "orc_write_treion"):
            getattr(_lib, fn).restype = C.c_size_t
            getattr(_lib, fn).argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        _lib.orc_read_restart.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                                          C.c_size_t]
        _lib.orc_cosmo_expansion.argtypes = [C.c_void_p, C.c_float, C.c_float]
        _lib.orc_set_subgrid.argtypes = [C.c_void_p] * 7 + [C.c_int]
        _lib.orc_hydro_step.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                        C.c_float]
        _lib.orc_set_tau_limit.argtypes = [C.c_void_p, C.c_double]
        _lib.orc_adj_objective.restype = C.c_double
        _lib.orc_adj_objective.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_long)]
    return _lib


def make_params(spec: W.BoxSpec, seed: int, path_length: int = 8) -> Params:
    p = Params()
    p.N = spec.n
    p.F = 5
    p.path_length = path_length
    p.itercount = 5
    p.ray_per_cell_max = spec.ray_per_cell_max
    p.hpx_lvl = 0
    for i, e in enumerate(W.NU_EV_5BIN):
        p.nu_eV[i] = e
    for i, a in enumerate(SPEC_ALPHA):
        p.spectrum_alpha[i] = a
    for r, vals in SPEC_ROWS.items():
        for nu, v in enumerate(vals):
            p.spectrum_table[r][nu] = v
    p.cl_factor = spec.cl_factor()
    p.box_hmpc = spec.box_hmpc
    p.z = spec.z
    p.const_clump = 1.0
    p.rkill_cm = spec.rkill_cm()
    p.seed = seed
    return p


class Oracle:
    """One box of the CPU restatement."""

    def __init__(self, inp: W.BoxInputs, seed: int):
        self._lib = lib()
        self.spec = inp.spec
        ijk, lum = W.grid_sources(inp)
        self._keep = [np.ascontiguousarray(inp.delta1, dtype=np.float32), np.ascontiguousarray(ijk, np.int32),
                      np.ascontiguousarray(lum, np.float64)]
        clump = None if inp.clump is None else np.ascontiguousarray(inp.clump, np.float32)
        self._keep.append(clump)
        self._p = make_params(inp.spec, seed)
        self.h = self._lib.orc_create(C.byref(self._p), self._keep[0].ctypes.data, len(lum),
                                      self._keep[1].ctypes.data, self._keep[2].ctypes.data,
                                      None if clump is None else clump.ctypes.data)

    def step(self) -> None:
        self._lib.orc_step(self.h)

    def num_rays(self) -> int:
        return int(self._lib.orc_num_rays(self.h))

    def last_crossings(self) -> int:
        return int(self._lib.orc_last_crossings(self.h))

    def scalars(self) -> np.ndarray:
        out = np.zeros(16, np.float64)
        self._lib.orc_scalars(self.h, out.ctypes.data)
        return out

    def adj_objective(self, lo, hi, lam=None, sc=None, dlam=None, dsc=None):
        """FP64 objective sum(Gamma_HI over [lo, hi)) of the next step as a function of source
        luminosity factors lam and per-cell density factors sc (frt_oracle.cc, orc_adj_objective),
        with its directional derivative along (dlam, dsc). Returns (J, dJ, lit cell count)."""
        lo = np.ascontiguousarray(lo, np.int32)
        hi = np.ascontiguousarray(hi, np.int32)
        keep = [None if v is None else np.ascontiguousarray(v, np.float64) for v in (lam, sc, dlam, dsc)]
        ptr = [None if v is None else v.ctypes.data for v in keep]
        jvp = C.c_double(0.0)
        nlit = C.c_long(0)
        J = self._lib.orc_adj_objective(self.h, lo.ctypes.data, hi.ctypes.data, ptr[0], ptr[1], ptr[2], ptr[3],
                                        C.byref(jvp), C.byref(nlit))
        return float(J), float(jvp.value), int(nlit.value)

    def cosmo_expansion(self, a_current: float, a_prev: float) -> None:
        """update_cosmo_expansion with the given scale factors, then update_dt."""
        self._lib.orc_cosmo_expansion(self.h, C.c_float(a_current), C.c_float(a_prev))

    def set_tau_limit(self, tau_max: float) -> None:
        """The opt-in optical-depth limit (not in the reference): a ray whose optical depth since
        its cast exceeds tau_max in every bin is removed after the step's last ray pass; the dump
        then carries each ray's HI and HeI columns ("ray_col"). 0 turns it off."""
        self._lib.orc_set_tau_limit(self.h, C.c_double(tau_max))

    def set_subgrid(self, tables, consts, ifront: bool = False) -> None:
        """The sub-grid model (equilibrium; with I-front tracking when ifront) with the
        reference's in-memory tables (tests/golden/subgrid_tables.reference_arrays) and
        cosmic-time constants {tinit, t(z=12), t(z=8), t(z=5.5), tre_dom[0..2]}."""
        keep = [np.ascontiguousarray(tables[k], np.float32) for k in ("time", "fh1", "t_dnl", "ds", "dnl")]
        c = np.ascontiguousarray(consts, np.float32)
        self._sg_keep = keep + [c]
        self._lib.orc_set_subgrid(self.h, *[a.ctypes.data for a in keep], c.ctypes.data, 1 if ifront else 0)

    def hydro_step(self, snap: W.BoxInputs, a_rt: float, dt_snap: float, zz: float) -> None:
        """update_hydro_step to the snapshot `snap` (its density and sources), then
        get_nphot_min_max and update_dt (frt_oracle.cc, orc_hydro_step)."""
        ijk, lum = W.grid_sources(snap)
        keep = [np.ascontiguousarray(snap.delta1, np.float32), np.ascontiguousarray(ijk, np.int32),
                np.ascontiguousarray(lum, np.float64)]
        self._lib.orc_hydro_step(self.h, keep[0].ctypes.data, len(lum), keep[1].ctypes.data, keep[2].ctypes.data,
                                 C.c_float(a_rt), C.c_float(dt_snap), C.c_float(zz))

    def _write(self, fn) -> bytes:
        f = getattr(self._lib, fn)
        n = f(self.h, None, 0)
        buf = (C.c_ubyte * n)()
        f(self.h, buf, n)
        return bytes(buf)

    def write_restart(self):
        """(gas, rays, treion) restart records in the reference's formats (frt_oracle.cc)."""
        return self._write("orc_write_gas"), self._write("orc_write_rays"), self._write("orc_write_treion")

    def read_restart(self, gas: bytes, treion: bytes, rays: bytes) -> None:
        st = self._lib.orc_read_restart(self.h, gas, len(gas), treion, len(treion), rays, len(rays))
        if st != 0:
            raise ValueError(f"orc_read_restart: malformed record set ({st})")

    def dump(self, path: str) -> None:
        if self._lib.orc_dump(self.h, path.encode()) != 0:
            raise IOError(path)

    def close(self) -> None:
        if self.h:
            self._lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
