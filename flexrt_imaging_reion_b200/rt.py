"""Host-side mirror of the reference's RT call surface over the C ABI.

The reference driver (main.cc) calls, per step, set_clump, set_clight, update_rays, find_avg_unu,
set_lmerge/set_merge_domain/get_num_thresh/count_rays/calc_nphot_merge, merge, split_rays,
update_thermal, new_rays, update_dt (main.cc:108-264), after a set-up of init, update_dt,
set_spectrum, init_rt, new_rays and get_nphot_min_max (main.cc:10-106). RTContext exposes the same
calls by the same names; `step()` runs the fused CUDA-graph form of one whole step.

Random rotations: the reference draws siRand(Ntheta) = rand() % 42875 from glibc's rand() once per
step in merge() (ray_tracing.cc:327) and once per source in init_rays (ray_tracing.cc:233), in that
order. Each box here keeps its own glibc random stream (srand(seed) + rand() semantics, through
glibc's reentrant initstate_r/random_r), so a box reproduces the draws of a one-box reference run.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _abi
from . import workloads as W

# set_spectrum (gas_funcs.cc:44-70) at alpha = 1.5 interpolates between the table rows alpha = 1.5
# and 1.75 of the reference's 5-bin spectrum table (input_files/spectrum_tables_5bins.txt) with
# weight 0; only those rows and the alpha column enter the arithmetic.
_SPEC_ALPHA = [-0.5 + 0.25 * i for i in range(15)]
_SPEC_ROWS = {8: [0.2, 0.2, 0.2, 0.2, 0.2], 9: [0.221, 0.213, 0.203, 0.191, 0.172]}


def spectrum_alpha15() -> np.ndarray:
    """set_spectrum() for the 5-bin table at alpha = 1.5, with the reference's float arithmetic."""
    a0, a1 = _SPEC_ALPHA[0], _SPEC_ALPHA[-1]
    m = int(np.floor((1.5 - a0) / (a1 - a0) * 14))
    m = min(m, 13)
    p = m + 1
    rows = _SPEC_ROWS
    spec = np.zeros(5, np.float32)
    ssum = np.float32(0.0)
    for nu in range(5):
        v = rows[m][nu] + (rows[p][nu] - rows[m][nu]) / (_SPEC_ALPHA[p] - _SPEC_ALPHA[m]) * (1.5 - _SPEC_ALPHA[m])
        spec[nu] = np.float32(v)
        ssum = np.float32(ssum + spec[nu])
    return (spec / ssum).astype(np.float32)


class RandStream:
    """glibc rand() sequence after srand(seed), kept per box with initstate_r / random_r."""

    _libc = None

    def __init__(self, seed: int):
        if RandStream._libc is None:
            RandStream._libc = C.CDLL("libc.so.6")
            RandStream._libc.initstate_r.argtypes = [C.c_uint, C.c_void_p, C.c_size_t, C.c_void_p]
            RandStream._libc.random_r.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
        self._state = C.create_string_buffer(128)
        self._data = C.create_string_buffer(64)
        if RandStream._libc.initstate_r(C.c_uint(seed), self._state, 128, self._data) != 0:
            raise RuntimeError("initstate_r failed")
        self._out = C.c_int32(0)

    def rand(self) -> int:
        RandStream._libc.random_r(self._data, C.byref(self._out))
        return int(self._out.value)

    def si_rand(self, a: int = _abi.FRT_NTHETA) -> int:
        return self.rand() % a


class FrtError(RuntimeError):
    pass


class RTContext:
    """One or more independent boxes of the RT step on one GPU."""

    def __init__(self, inputs: Sequence[W.BoxInputs], seeds: Sequence[int], precision: str = "mixed",
                 outputs: str = "core", ray_capacity: Optional[int] = None, lit_capacity: int = 0,
                 device: int = 0, path_length: int = 8):
        self.L = _abi.lib()
        self.inputs = list(inputs)
        self.specs = [i.spec for i in self.inputs]
        self.nbox = len(self.inputs)
        self.F = 5
        self.spectrum = spectrum_alpha15()
        self._boxes = (_abi.BoxDesc * self.nbox)()
        for b, s in enumerate(self.specs):
            bd = self._boxes[b]
            bd.n = s.n
            bd.box_hmpc = s.box_hmpc
            bd.zz = s.z
            bd.cl_factor = s.cl_factor()
            bd.ray_per_cell_max = s.ray_per_cell_max
            bd.rkill_cm = s.rkill_cm()
        cfg = _abi.Config()
        cfg.nfreq = self.F
        for nu, e in enumerate(W.NU_EV_5BIN):
            cfg.nu_phot[nu] = e / W.H_EV
            cfg.spectrum[nu] = float(self.spectrum[nu])
        cfg.itercount = 5
        self.itercount = cfg.itercount
        cfg.path_length = path_length
        cfg.hpx_lvl = 0
        cfg.safety_factor = 3.0
        cfg.tstep_factor = 1.0
        cfg.nl_const = 0.5
        cfg.const_clump = 1.0
        cfg.fH1_0 = 1.0 - 1.2e-3
        cfg.fHe1_0 = 1.0 - 1.2e-3
        cfg.fHe2_0 = 1.2e-3
        cfg.temp_0 = 1e4
        cfg.nbox = self.nbox
        cfg.boxes = C.cast(self._boxes, C.POINTER(_abi.BoxDesc))
        ncell = sum(s.n ** 3 for s in self.specs)
        cfg.ray_capacity = int(ray_capacity or max(1 << 20, 4 * ncell))
        cfg.lit_capacity = int(lit_capacity)
        self.src = [W.grid_sources(i) for i in self.inputs]
        cfg.src_capacity = max(1, sum(len(l) for _, l in self.src))
        cfg.precision = _abi.FRT_PREC_STRICT if precision == "strict" else _abi.FRT_PREC_MIXED
        cfg.outputs = _abi.FRT_OUT_DIAG if outputs == "diag" else _abi.FRT_OUT_CORE
        cfg.device = device
        self._cfg = cfg
        h = C.c_void_p()
        st = self.L.frt_create(C.byref(cfg), C.byref(h))
        self.h = h
        self._check(st, "frt_create")
        self.nsrc_box = [len(l) for _, l in self.src]
        self.nsrc = sum(self.nsrc_box)
        self._ith_box = np.zeros(self.nbox, np.uint16)
        self._ith_src = np.zeros(max(1, self.nsrc), np.uint16)
        self.stats = _abi.StepStats()
        seeds_arr = np.ascontiguousarray([int(s) & 0xFFFFFFFF for s in seeds], np.uint32)
        self._check(self.L.frt_seed_boxes(self.h, seeds_arr.ctypes.data), "frt_seed_boxes")

    # ---- plumbing ---------------------------------------------------------------------------
    def _check(self, st: int, what: str) -> None:
        if st != _abi.FRT_OK:
            msg = self.L.frt_last_error(self.h).decode() if self.h else ""
            raise FrtError(f"{what} failed with status {st}: {msg}")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.frt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- set-up, as main.cc:10-106 -------------------------------------------------------------
    def setup(self, owner=None) -> None:
        """init + init_rt + the set-up cast + get_nphot_min_max. With `owner` (one byte per
        source, in set-up order), only the sources marked 1 are cast, here and in every step
        (frt_set_source_owner): the context then holds one share of a box's sources."""
        for b, inp in enumerate(self.inputs):
            d1 = np.ascontiguousarray(inp.delta1, np.float32)
            self._check(self.L.frt_init_gas(self.h, b, d1.ctypes.data), "frt_init_gas")
            ijk, lum = self.src[b]
            ijk = np.ascontiguousarray(ijk, np.int32)
            lum = np.ascontiguousarray(lum, np.float64)
            self._check(self.L.frt_set_sources(self.h, b, len(lum), ijk.ctypes.data, lum.ctypes.data),
                        "frt_set_sources")
            if inp.clump is not None:
                cl = np.ascontiguousarray(inp.clump, np.float32)
                self._check(self.L.frt_set_clump_field(self.h, b, cl.ctypes.data), "frt_set_clump_field")
        if owner is not None:
            own = np.ascontiguousarray(owner, np.uint8)
            self._check(self.L.frt_set_source_owner(self.h, own.ctypes.data), "frt_set_source_owner")
        self.update_dt()
        self.init_rt()
        self.new_rays(self.draw_cast())
        self.get_nphot_min_max()

    def step_phase(self, phase: int, it: int = 0) -> Dict[str, float]:
        """frt_step_phase: one phase of a step shared with other contexts (partition.py)."""
        self._check(self.L.frt_step_phase(self.h, phase, it, None, None, C.byref(self.stats)), "frt_step_phase")
        return self.stats.as_dict()

    def set_phase_async(self, on: bool) -> None:
        """frt_set_phase_async: phases only enqueue on the context's stream (phase_stream())."""
        self._check(self.L.frt_set_phase_async(self.h, int(bool(on))), "frt_set_phase_async")

    def phase_stream(self) -> int:
        """The context's stream (cudaStream_t as an integer), for work ordered with the phases."""
        v = C.c_void_p()
        self._check(self.L.frt_phase_stream(self.h, C.byref(v)), "frt_phase_stream")
        return int(v.value or 0)

    def phase_buffers(self):
        """Device addresses and sizes of the arrays combined between phases:
        (lit_flag, ncell, lit_acc, lit_heat, nlit)."""
        lf, la, lh = C.c_void_p(), C.c_void_p(), C.c_void_p()
        nc, nl = C.c_longlong(), C.c_longlong()
        self._check(self.L.frt_phase_buffers(self.h, C.byref(lf), C.byref(nc), C.byref(la), C.byref(lh), C.byref(nl)),
                    "frt_phase_buffers")
        return lf.value, nc.value, la.value, lh.value, nl.value

    def setup_restart(self, files) -> None:
        """Set-up from restart records in the reference's formats, one (gas, treion, rays) bytes
        triple per box (the reference's restart path: init() and init_rt() with input_grid = TRUE,
        no set-up cast)."""
        for b, (gas, tre, _) in enumerate(files):
            self._check(self.L.frt_read_gas(self.h, b, gas, len(gas)), "frt_read_gas")
            self._check(self.L.frt_read_treion(self.h, b, tre, len(tre)), "frt_read_treion")
            ijk, lum = self.src[b]
            ijk = np.ascontiguousarray(ijk, np.int32)
            lum = np.ascontiguousarray(lum, np.float64)
            self._check(self.L.frt_set_sources(self.h, b, len(lum), ijk.ctypes.data, lum.ctypes.data),
                        "frt_set_sources")
            inp = self.inputs[b]
            if inp.clump is not None:
                cl = np.ascontiguousarray(inp.clump, np.float32)
                self._check(self.L.frt_set_clump_field(self.h, b, cl.ctypes.data), "frt_set_clump_field")
        self.update_dt()
        self.init_rt()
        for b, (_, _, rays) in enumerate(files):
            self._check(self.L.frt_read_rays(self.h, b, rays, len(rays)), "frt_read_rays")
        self.get_nphot_min_max()

    def set_cast_per_source(self, on: bool) -> None:
        """One cast launch per source in step(graph=False) (the unbatched comparison form)."""
        self._check(self.L.frt_set_cast_per_source(self.h, int(bool(on))), "frt_set_cast_per_source")

    def cosmo_expansion(self, a_current, a_prev) -> None:
        """update_cosmo_expansion + update_dt with per-box scale factors (end and start of the
        step just taken)."""
        ac = np.ascontiguousarray(np.broadcast_to(np.asarray(a_current, np.float32), (self.nbox,)))
        ap = np.ascontiguousarray(np.broadcast_to(np.asarray(a_prev, np.float32), (self.nbox,)))
        self._check(self.L.frt_update_cosmo_expansion(self.h, ac.ctypes.data, ap.ctypes.data),
                    "frt_update_cosmo_expansion")

    def set_subgrid(self, tables, consts, ifront: bool = False) -> None:
        """frt_set_subgrid: the sub-grid RadHydro model from here on, with I-front tracking when
        `ifront`. `tables` holds the reference's in-memory arrays ("time", "fh1": Nt*27+1 floats;
        "t_dnl", "ds": 500; "dnl": 500*500), `consts` the cosmic times (tinit, t(z=12), t(z=8),
        t(z=5.5), tre_dom[0..2])."""
        keep = {k: np.ascontiguousarray(tables[k], np.float32) for k in ("time", "fh1", "t_dnl", "ds", "dnl")}
        t = _abi.SubgridTables()
        t.time_RH, t.fh1_RH = keep["time"].ctypes.data, keep["fh1"].ctypes.data
        t.t_deltaNL, t.delta_over_sigma, t.deltaNL = keep["t_dnl"].ctypes.data, keep["ds"].ctypes.data, keep["dnl"].ctypes.data
        c = [float(x) for x in consts]
        t.tinit, t.t_z12, t.t_z8, t.t_z55 = c[0], c[1], c[2], c[3]
        for k in range(3):
            t.tre_dom[k] = c[4 + k]
        t.ifront = 1 if ifront else 0
        self._check(self.L.frt_set_subgrid(self.h, C.byref(t)), "frt_set_subgrid")

    def hydro_step(self, box: int, snap: W.BoxInputs, a_rt: float, dt_snap: float, zz: float) -> None:
        """update_hydro_step of one box to the snapshot `snap` (its density cube and sources), with
        get_nphot_min_max; call after new_rays and the expansion, as main.cc:219-222 does."""
        d1 = np.ascontiguousarray(snap.delta1, np.float32)
        ijk, lum = W.grid_sources(snap)
        ijk = np.ascontiguousarray(ijk, np.int32)
        lum = np.ascontiguousarray(lum, np.float64)
        self._check(self.L.frt_update_hydro_step(self.h, box, d1.ctypes.data, C.c_float(a_rt), C.c_float(dt_snap),
                                                 C.c_float(zz), len(lum), ijk.ctypes.data, lum.ctypes.data),
                    "frt_update_hydro_step")
        self.src[box] = (ijk, lum)
        self.nsrc_box[box] = len(lum)
        self.nsrc = sum(self.nsrc_box)

    def write_restart(self, box: int = 0):
        """(gas, rays, treion) records of a box in the reference's restart formats."""
        out = []
        for fn in ("frt_write_gas", "frt_write_rays", "frt_write_treion"):
            n = C.c_size_t(0)
            self._check(getattr(self.L, fn)(self.h, box, None, 0, C.byref(n)), fn)
            buf = (C.c_ubyte * n.value)()
            self._check(getattr(self.L, fn)(self.h, box, buf, n.value, C.byref(n)), fn)
            out.append(bytes(buf))
        return tuple(out)

    def draw_cast(self) -> np.ndarray:
        """init_rays draws of the set-up cast, from the context's per-box glibc streams."""
        out = np.zeros(max(1, self.nsrc), np.uint16)
        self._check(self.L.frt_draw_cast(self.h, out.ctypes.data), "frt_draw_cast")
        return out

    def draw_step(self):
        """Draws of one step in reference order: merge() first, then init_rays per source."""
        m = np.zeros(self.nbox, np.uint16)
        c = np.zeros(max(1, self.nsrc), np.uint16)
        self._check(self.L.frt_draw_step(self.h, m.ctypes.data, c.ctypes.data), "frt_draw_step")
        return m, c

    # ---- the reference's step functions ---------------------------------------------------------
    def update_dt(self) -> np.ndarray:
        dt = np.zeros(self.nbox, np.float32)
        self._check(self.L.frt_update_dt(self.h, dt.ctypes.data), "frt_update_dt")
        return dt

    def init_rt(self) -> None:
        self._check(self.L.frt_init_rt(self.h), "frt_init_rt")

    def get_nphot_min_max(self):
        mn = np.zeros(self.nbox)
        mx = np.zeros(self.nbox)
        self._check(self.L.frt_get_nphot_min_max(self.h, mn.ctypes.data, mx.ctypes.data), "frt_get_nphot_min_max")
        return mn, mx

    def set_clump(self) -> None:
        self._check(self.L.frt_set_clump(self.h), "frt_set_clump")

    def set_clight(self) -> None:
        self._check(self.L.frt_set_clight(self.h), "frt_set_clight")

    def update_rays(self) -> None:
        self._check(self.L.frt_update_rays(self.h), "frt_update_rays")

    def find_avg_unu(self) -> None:
        self._check(self.L.frt_find_avg_unu(self.h), "frt_find_avg_unu")

    def count_rays(self) -> np.ndarray:
        out = np.zeros(self.nbox, np.int64)
        self._check(self.L.frt_count_rays(self.h, out.ctypes.data), "frt_count_rays")
        return out

    def merge(self, itheta_per_box: np.ndarray) -> None:
        a = np.ascontiguousarray(itheta_per_box, np.uint16)
        self._check(self.L.frt_merge(self.h, a.ctypes.data), "frt_merge")

    def split_rays(self) -> None:
        self._check(self.L.frt_split_rays(self.h), "frt_split_rays")

    def update_thermal(self) -> None:
        self._check(self.L.frt_update_thermal(self.h), "frt_update_thermal")

    def new_rays(self, itheta_per_source: np.ndarray) -> None:
        a = np.ascontiguousarray(itheta_per_source, np.uint16)
        self._check(self.L.frt_new_rays(self.h, a.ctypes.data), "frt_new_rays")

    # ---- whole steps ------------------------------------------------------------------------------
    def step_unfused(self) -> None:
        """One step through the individual step functions, in main.cc's order."""
        self.set_clump()
        self.set_clight()
        self.update_rays()
        self.find_avg_unu()
        m, c = self.draw_step()
        self.merge(m)
        self.split_rays()
        self.update_thermal()
        self.new_rays(c)
        self.update_dt()

    def step(self, graph: bool = True, draws=None) -> Dict[str, float]:
        """One whole step, fused (CUDA graph when graph=True). Without `draws` the library draws
        the step's random angles from its per-box streams (reference order)."""
        fn = self.L.frt_step if graph else self.L.frt_step_plain
        if draws is None:
            st = fn(self.h, None, None, C.byref(self.stats))
        else:
            m, c = draws
            self._ith_box[:] = m
            self._ith_src[: len(c)] = c[: len(self._ith_src)]
            st = fn(self.h, self._ith_box.ctypes.data, self._ith_src.ctypes.data, C.byref(self.stats))
        self._check(st, "frt_step")
        return self.stats.as_dict()

    # ---- launch shapes -------------------------------------------------------------------------
    def autotune(self, steps: int = 4) -> Dict[str, float]:
        """frt_autotune: `steps` RT steps that also time candidate launch shapes; the chosen
        shapes are set on the context (and remembered for its ray-count bucket)."""
        t = _abi.Tuning()
        self._check(self.L.frt_autotune(self.h, int(steps), C.byref(t)), "frt_autotune")
        return t.as_dict()

    def tuning(self) -> Dict[str, float]:
        t = _abi.Tuning()
        self._check(self.L.frt_get_tuning(self.h, C.byref(t)), "frt_get_tuning")
        return t.as_dict()

    def set_tuning(self, **shape) -> None:
        """frt_set_tuning with the given fields changed from the current shapes."""
        t = _abi.Tuning()
        self._check(self.L.frt_get_tuning(self.h, C.byref(t)), "frt_get_tuning")
        for k, v in shape.items():
            setattr(t, k, v)
        self._check(self.L.frt_set_tuning(self.h, C.byref(t)), "frt_set_tuning")

    def last_stats(self) -> Dict[str, float]:
        st = _abi.StepStats()
        self._check(self.L.frt_last_stats(self.h, C.byref(st)), "frt_last_stats")
        return st.as_dict()

    def in_flight(self) -> float:
        """Photons in the live rays (the running total of the device ledger)."""
        return float(self.last_stats()["photons_in_flight"])

    def last_timing(self):
        a = C.c_float(0.0)
        b = C.c_float(0.0)
        self._check(self.L.frt_last_timing(self.h, C.byref(a), C.byref(b)), "frt_last_timing")
        return a.value, b.value

    # ---- state access --------------------------------------------------------------------------------
    def get_field(self, box: int, name: str) -> np.ndarray:
        n = self.specs[box].n
        shape = (n ** 3, self.F) if name in _abi.PER_BIN_FIELDS else ((n ** 3, 10) if name == "TCROSS_NEW" else (n ** 3,))
        out = np.zeros(shape, np.float32)
        self._check(self.L.frt_get_field(self.h, box, _abi.FIELD_ID[name], out.ctypes.data), f"get_field {name}")
        return out

    def set_field(self, box: int, name: str, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, np.float32)
        self._check(self.L.frt_set_field(self.h, box, _abi.FIELD_ID[name], a.ctypes.data), f"set_field {name}")

    def num_rays(self, box: int = -1) -> int:
        n = C.c_longlong(0)
        self._check(self.L.frt_num_rays(self.h, box, C.byref(n)), "frt_num_rays")
        return int(n.value)

    def rays(self, box: int = 0) -> Dict[str, np.ndarray]:
        n = self.num_rays(box)
        out = {"ray_order": np.zeros(n, np.int16), "ray_pixel": np.zeros(n, np.int32),
               "ray_itheta": np.zeros(n, np.uint16), "ray_cell": np.zeros(n, np.int32),
               "ray_geom": np.zeros((n, 9), np.float32), "ray_nphot": np.zeros((n, self.F), np.float32)}
        self._check(self.L.frt_download_rays(self.h, box, out["ray_order"].ctypes.data, out["ray_pixel"].ctypes.data,
                                             out["ray_itheta"].ctypes.data, out["ray_cell"].ctypes.data,
                                             out["ray_geom"].ctypes.data, out["ray_nphot"].ctypes.data),
                    "frt_download_rays")
        return out

    def set_tau_limit(self, tau_max: float) -> None:
        """frt_set_tau_limit: remove rays whose optical depth since their cast exceeds tau_max in
        every frequency bin (an opt-in rule the reference does not have; 0 turns it off)."""
        self._check(self.L.frt_set_tau_limit(self.h, C.c_double(tau_max)), "frt_set_tau_limit")

    def ray_columns(self, box: int = 0) -> np.ndarray:
        """The HI and HeI column densities (cm^-2) of the live rays, [n, 2] float64, in the order
        of rays()."""
        n = self.num_rays(box)
        out = np.zeros((n, 2), np.float64)
        self._check(self.L.frt_download_ray_columns(self.h, box, out.ctypes.data), "frt_download_ray_columns")
        return out

    def adjoint(self, lo, hi, box: int = 0, want_dl: bool = True, want_dnh: bool = True):
        """frt_adjoint: J = sum of Gamma_HI over cells [lo, hi) of `box` after the next step's
        C2Ray iteration, with dJ/dL per source (photons/s) and dJ/dn_H per cell (cm^-3, N^3).
        Needs the state right after setup()."""
        obj = _abi.AdjObjective()
        obj.box = box
        for k in range(3):
            obj.lo[k] = int(lo[k])
            obj.hi[k] = int(hi[k])
        J = C.c_double(0.0)
        dl = np.zeros(max(1, self.nsrc_box[box]), np.float64) if want_dl else None
        dnh = np.zeros(self.specs[box].n ** 3, np.float32) if want_dnh else None
        self._check(self.L.frt_adjoint(self.h, C.byref(obj), C.byref(J), None if dl is None else dl.ctypes.data,
                                       None if dnh is None else dnh.ctypes.data), "frt_adjoint")
        if dl is not None:
            dl = dl[:self.nsrc_box[box]]
        return float(J.value), dl, dnh

    def last_raypass_ms(self) -> float:
        """Device time of the ray passes of the last step (sum over the C2Ray iterations)."""
        v = C.c_float(0.0)
        self._check(self.L.frt_last_kernel_timing(self.h, 1, C.byref(v)), "frt_last_kernel_timing")
        return float(v.value)

    def last_walk_ms(self) -> float:
        """Device time of the walk (k_advance over every live ray) of the last step."""
        v = C.c_float(0.0)
        self._check(self.L.frt_last_kernel_timing(self.h, 2, C.byref(v)), "frt_last_kernel_timing")
        return float(v.value)

    def last_adjoint_ms(self) -> float:
        v = C.c_float(0.0)
        self._check(self.L.frt_last_adjoint_timing(self.h, C.byref(v)), "frt_last_adjoint_timing")
        return float(v.value)

    def take_rays(self, box: int = 0, in_step: bool = False) -> bytes:
        """frt_take_rays: the live rays of the box as ray records (bytes); the context keeps none.
        in_step: between the step's last C2Ray pass and its end phase (the pass's removals are
        skipped); otherwise between steps."""
        n = C.c_size_t(0)
        self._check(self.L.frt_take_rays(self.h, box, 1 if in_step else 0, None, 0, C.byref(n)), "frt_take_rays")
        buf = C.create_string_buffer(n.value)
        self._check(self.L.frt_take_rays(self.h, box, 1 if in_step else 0, buf, n.value, C.byref(n)),
                    "frt_take_rays")
        return buf.raw[: n.value]

    def put_rays(self, data: bytes, box: int = 0) -> None:
        """frt_put_rays: appends ray records taken from another context of the same box."""
        self._check(self.L.frt_put_rays(self.h, box, data, len(data)), "frt_put_rays")

    def set_nphot_merge(self, value: float, box: int = 0) -> None:
        self._check(self.L.frt_set_nphot_merge(self.h, box, C.c_double(value)), "frt_set_nphot_merge")

    def box_scalars(self, box: int = 0) -> Dict[str, float]:
        v = np.zeros(8)
        self._check(self.L.frt_box_scalars(self.h, box, v.ctypes.data), "frt_box_scalars")
        keys = ["t", "dt", "nphot_min", "nphot_max", "nphot_merge", "num_thresh", "dx", "dx0"]
        return dict(zip(keys, v.tolist()))

    def rotation_table(self) -> np.ndarray:
        out = np.zeros((_abi.FRT_NTHETA, 18), np.float32)
        self._check(self.L.frt_rotation_table(self.h, out.ctypes.data), "frt_rotation_table")
        return out
