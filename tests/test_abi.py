"""The C-ABI library: it loads, exports every entry point include/flexrt.h declares, and fails with a
status (never a crash) when no CUDA device is usable."""
import ctypes as C
import os
import re

import numpy as np

from flexrt_imaging_reion_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def declared_symbols():
    txt = open(os.path.join(REPO, "include", "flexrt.h")).read()
    return sorted(set(re.findall(r"^\s*(?:frt_status|const char\*)\s+(frt_\w+)\s*\(", txt, flags=re.M)))


def test_exports_every_declared_symbol(product_lib):
    syms = declared_symbols()
    assert len(syms) >= 28
    for s in syms:
        assert hasattr(product_lib, s), s
    assert set(syms) <= set(_abi.EXPORTS) | {"frt_build_rotation_table"}


def test_struct_layouts_match_header():
    # field order / sizes of the ctypes mirrors (x86-64 ABI)
    assert C.sizeof(_abi.BoxDesc) == 40
    assert C.sizeof(_abi.StepStats) == 8 * 8 + 7 * 8 + 8
    assert _abi.Config.boxes.offset % 8 == 0


def test_invalid_config_rejected(product_lib):
    cfg = _abi.Config()   # nbox = 0
    h = C.c_void_p()
    assert product_lib.frt_create(C.byref(cfg), C.byref(h)) == _abi.FRT_ERR_INVALID


def test_null_context_calls_fail_cleanly(product_lib):
    for name in ("frt_update_rays", "frt_find_avg_unu", "frt_split_rays", "frt_update_thermal", "frt_init_rt"):
        assert getattr(product_lib, name)(None) == _abi.FRT_ERR_INVALID
    assert product_lib.frt_set_source_owner(None, None) == _abi.FRT_ERR_INVALID
    assert product_lib.frt_step_phase(None, _abi.PHASE_WALK, 0, None, None, None) == _abi.FRT_ERR_INVALID
    assert product_lib.frt_phase_buffers(None, None, None, None, None, None) == _abi.FRT_ERR_INVALID
