"""ctypes declarations of the C ABI in include/flexrt.h (libflexrt_b200.so).

The library is loaded from the package's lib/ directory; importing this module fails loudly when
it is missing -- there is no CPU fallback for the RT path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libflexrt_b200.so")

FRT_MAX_FREQ = 8
FRT_NTHETA = 42875

FRT_OK, FRT_ERR_INVALID, FRT_ERR_CAPACITY, FRT_ERR_TIMEOUT, FRT_ERR_CUDA, FRT_ERR_STATE = range(6)
FRT_PREC_MIXED, FRT_PREC_STRICT = 0, 1
FRT_OUT_CORE, FRT_OUT_DIAG = 0, 1

FIELDS = ["RHO", "NH", "NHE", "NH1", "NHE1", "NH2", "NHE2", "NE", "N_TOT", "F_H1", "F_HE1", "F_H2", "F_HE2", "TEMP",
          "CLUMP", "AVG_NH1", "AVG_NHE1", "GAMMA_H1_TOT", "GAMMA_HE1_TOT", "HEAT_RATE", "COOL_RATE", "TREION",
          "TREION_FLAG", "DNE_DT", "RECOMB_H2", "RECOMB_HE2", "RECRATE_H2", "RECRATE_HE2", "MFP", "MFP_912",
          "IF_SPEED", "INC_FLUX", "GAMMA_H1_NU", "GAMMA_HE1_NU", "NGAM_NU", "U_NU", "FION", "FION_MAX", "TCROSS",
          "DELTA_FION", "TREION_OUT", "TCROSS_FLAG", "NEUTRAL_FLAG", "TCROSS_NEW"]
FIELD_ID = {name: i for i, name in enumerate(FIELDS)}
PER_BIN_FIELDS = {"GAMMA_H1_NU", "GAMMA_HE1_NU", "NGAM_NU", "U_NU"}

EXPORTS = ["frt_create", "frt_destroy", "frt_last_error", "frt_rotation_table", "frt_build_rotation_table", "frt_init_gas", "frt_set_sources",
           "frt_set_clump_field", "frt_set_field", "frt_get_field", "frt_init_rt", "frt_update_dt",
           "frt_get_nphot_min_max", "frt_set_clump", "frt_set_clight", "frt_update_rays", "frt_find_avg_unu",
           "frt_count_rays", "frt_merge", "frt_split_rays", "frt_update_thermal", "frt_new_rays", "frt_step",
           "frt_step_plain", "frt_last_stats", "frt_num_rays", "frt_download_rays", "frt_box_scalars",
           "frt_last_timing", "frt_seed_boxes", "frt_draw_cast", "frt_draw_step", "frt_get_sparse_field_noalloc", "frt_adjoint",
           "frt_last_adjoint_timing", "frt_write_gas", "frt_write_rays", "frt_write_treion", "frt_read_gas",
           "frt_read_treion", "frt_read_rays", "frt_update_cosmo_expansion",
           "frt_set_cast_per_source", "frt_last_kernel_timing", "frt_set_source_owner", "frt_step_phase",
           "frt_phase_buffers", "frt_autotune", "frt_get_tuning", "frt_set_tuning", "frt_update_hydro_step", "frt_set_phase_async",
           "frt_phase_stream", "frt_set_subgrid", "frt_set_tau_limit", "frt_download_ray_columns", "frt_take_rays", "frt_put_rays", "frt_set_nphot_merge"]
PHASE_WALK, PHASE_CELLS, PHASE_RAYPASS, PHASE_CELLPASS, PHASE_END = 0, 1, 2, 3, 4
NOALLOC_MAX_CELLS = 1 << 20


class AdjObjective(C.Structure):
    _fields_ = [("box", C.c_int), ("lo", C.c_int * 3), ("hi", C.c_int * 3)]


class BoxDesc(C.Structure):
    _fields_ = [("n", C.c_int), ("box_hmpc", C.c_double), ("zz", C.c_float), ("cl_factor", C.c_float),
                ("ray_per_cell_max", C.c_int), ("rkill_cm", C.c_double)]


class Config(C.Structure):
    _fields_ = [("nfreq", C.c_int), ("nu_phot", C.c_double * FRT_MAX_FREQ), ("spectrum", C.c_float * FRT_MAX_FREQ),
                ("itercount", C.c_int), ("path_length", C.c_int), ("hpx_lvl", C.c_int),
                ("safety_factor", C.c_float), ("tstep_factor", C.c_float), ("nl_const", C.c_float),
                ("const_clump", C.c_float), ("fH1_0", C.c_float), ("fHe1_0", C.c_float), ("fHe2_0", C.c_float),
                ("temp_0", C.c_float), ("nbox", C.c_int), ("boxes", C.POINTER(BoxDesc)),
                ("ray_capacity", C.c_longlong), ("lit_capacity", C.c_longlong), ("src_capacity", C.c_longlong),
                ("precision", C.c_int), ("outputs", C.c_int), ("device", C.c_int)]


class Tuning(C.Structure):
    _fields_ = [("raypass_block", C.c_int), ("raypass_blocks_per_sm", C.c_int), ("raypass_chunk", C.c_int),
                ("walk_block", C.c_int), ("walk_blocks_per_sm", C.c_int), ("cellpass_blocks_per_sm", C.c_int),
                ("split_blocks_per_sm", C.c_int), ("steps", C.c_int), ("raypass_ns_per_crossing", C.c_double),
                ("walk_ns_per_ray", C.c_double), ("cellpass_ns_per_cell", C.c_double),
                ("split_ns_per_ray", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SubgridTables(C.Structure):
    _fields_ = [("time_RH", C.c_void_p), ("fh1_RH", C.c_void_p), ("t_deltaNL", C.c_void_p),
                ("delta_over_sigma", C.c_void_p), ("deltaNL", C.c_void_p), ("tinit", C.c_float),
                ("t_z12", C.c_float), ("t_z8", C.c_float), ("t_z55", C.c_float), ("tre_dom", C.c_float * 3),
                ("ifront", C.c_int)]


class StepStats(C.Structure):
    _fields_ = [("rays_alive", C.c_longlong), ("rays_moved", C.c_longlong), ("crossings", C.c_longlong),
                ("lit_cells", C.c_longlong), ("rays_split", C.c_longlong), ("rays_merged", C.c_longlong),
                ("rays_killed", C.c_longlong), ("rays_cast", C.c_longlong), ("photons_emitted", C.c_double),
                ("photons_deposited", C.c_double), ("photons_killed", C.c_double), ("photons_overlap", C.c_double),
                ("photons_in_flight", C.c_double), ("t", C.c_double), ("dt", C.c_double),
                ("error_flags", C.c_uint), ("pad", C.c_uint)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with flexrt_imaging_reion_b200.build.build() "
                           "(the RT step has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    P, I, LL, U16P = C.c_void_p, C.c_int, C.c_longlong, C.c_void_p
    sig = {
        "frt_create": ([C.POINTER(Config), C.POINTER(C.c_void_p)], I),
        "frt_destroy": ([P], I),
        "frt_last_error": ([P], C.c_char_p),
        "frt_rotation_table": ([P, P], I),
        "frt_build_rotation_table": ([P], I),
        "frt_init_gas": ([P, I, P], I),
        "frt_set_sources": ([P, I, I, P, P], I),
        "frt_set_clump_field": ([P, I, P], I),
        "frt_set_field": ([P, I, I, P], I),
        "frt_get_field": ([P, I, I, P], I),
        "frt_init_rt": ([P], I),
        "frt_update_dt": ([P, P], I),
        "frt_get_nphot_min_max": ([P, P, P], I),
        "frt_set_clump": ([P], I),
        "frt_set_clight": ([P], I),
        "frt_update_rays": ([P], I),
        "frt_find_avg_unu": ([P], I),
        "frt_count_rays": ([P, P], I),
        "frt_merge": ([P, U16P], I),
        "frt_split_rays": ([P], I),
        "frt_update_thermal": ([P], I),
        "frt_new_rays": ([P, U16P], I),
        "frt_step": ([P, U16P, U16P, C.POINTER(StepStats)], I),
        "frt_step_plain": ([P, U16P, U16P, C.POINTER(StepStats)], I),
        "frt_last_stats": ([P, C.POINTER(StepStats)], I),
        "frt_num_rays": ([P, I, C.POINTER(LL)], I),
        "frt_download_rays": ([P, I, P, P, P, P, P, P], I),
        "frt_set_tau_limit": ([P, C.c_double], I),
        "frt_take_rays": ([P, I, I, P, C.c_size_t, C.POINTER(C.c_size_t)], I),
        "frt_put_rays": ([P, I, P, C.c_size_t], I),
        "frt_set_nphot_merge": ([P, I, C.c_double], I),
        "frt_download_ray_columns": ([P, I, P], I),
        "frt_box_scalars": ([P, I, P], I),
        "frt_last_timing": ([P, P, P], I),
        "frt_seed_boxes": ([P, P], I),
        "frt_draw_cast": ([P, P], I),
        "frt_draw_step": ([P, P, P], I),
        "frt_get_sparse_field_noalloc": ([P, I, I, I, LL, LL, P], I),
        "frt_adjoint": ([P, C.POINTER(AdjObjective), P, P, P], I),
        "frt_last_adjoint_timing": ([P, P], I),
        "frt_write_gas": ([P, I, P, C.c_size_t, C.POINTER(C.c_size_t)], I),
        "frt_write_rays": ([P, I, P, C.c_size_t, C.POINTER(C.c_size_t)], I),
        "frt_write_treion": ([P, I, P, C.c_size_t, C.POINTER(C.c_size_t)], I),
        "frt_read_gas": ([P, I, P, C.c_size_t], I),
        "frt_read_treion": ([P, I, P, C.c_size_t], I),
        "frt_read_rays": ([P, I, P, C.c_size_t], I),
        "frt_update_cosmo_expansion": ([P, P, P], I),
        "frt_set_cast_per_source": ([P, I], I),
        "frt_set_source_owner": ([P, P], I),
        "frt_step_phase": ([P, I, I, P, P, C.POINTER(StepStats)], I),
        "frt_phase_buffers": ([P, C.POINTER(P), C.POINTER(LL), C.POINTER(P), C.POINTER(P), C.POINTER(LL)], I),
        "frt_last_kernel_timing": ([P, I, P], I),
        "frt_autotune": ([P, I, C.POINTER(Tuning)], I),
        "frt_update_hydro_step": ([P, I, P, C.c_float, C.c_float, C.c_float, I, P, P], I),
        "frt_set_phase_async": ([P, I], I),
        "frt_set_subgrid": ([P, C.POINTER(SubgridTables)], I),
        "frt_phase_stream": ([P, C.POINTER(P)], I),
        "frt_get_tuning": ([P, C.POINTER(Tuning)], I),
        "frt_set_tuning": ([P, C.POINTER(Tuning)], I),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L
