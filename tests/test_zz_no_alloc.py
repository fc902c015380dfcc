"""frt_get_sparse_field_noalloc: the lit-cell field read-back through the library's static
scratch array (no device allocation) returns what frt_get_field returns.

Collected last on purpose: the first call on a device looks up the scratch address, and the test
must pass both in a fresh process (first call here) and after every other test ran.
"""
import ctypes as C

import numpy as np
import pytest

from flexrt_imaging_reion_b200 import _abi, rt, workloads as W

pytestmark = pytest.mark.gpu


def _noalloc(ctx, box, field, bin_, first, count):
    out = np.zeros(count, np.float32)
    st = ctx.L.frt_get_sparse_field_noalloc(ctx.h, box, _abi.FIELD_ID[field], bin_, first, count,
                                            out.ctypes.data)
    return st, out


def _read_windows(ctx, box, field, bin_, ncell, window):
    out = np.zeros(ncell, np.float32)
    for first in range(0, ncell, window):
        count = min(window, ncell - first)
        st, part = _noalloc(ctx, box, field, bin_, first, count)
        assert st == _abi.FRT_OK, ctx.L.frt_last_error(ctx.h).decode()
        out[first:first + count] = part
    return out


@pytest.mark.parametrize("outputs", ["diag", "core"])
def test_noalloc_matches_get_field_twice(outputs):
    spec = W.config_tiny(n=32, n_src=12, steps=3, seed=7, name="T32")
    ctx = rt.RTContext([W.make_inputs(spec)], [3], outputs=outputs, ray_capacity=1 << 20)
    ctx.setup()
    ncell = spec.n ** 3
    fields = [("GAMMA_H1_TOT", 0), ("GAMMA_HE1_TOT", 0)]
    if outputs == "diag":
        fields += [("NGAM_NU", 2), ("GAMMA_H1_NU", 1), ("GAMMA_HE1_NU", 4)]
    for _ in range(2):   # two calls in a row, each after a step
        ctx.step()
        for field, b in fields:
            ref = ctx.get_field(0, field)
            if ref.ndim == 2:
                ref = ref[:, b]
            got = _read_windows(ctx, 0, field, b, ncell, 5000)
            # same gather kernel and the same lit-cell values: equal to the last bit
            np.testing.assert_array_equal(got, ref)
            assert field == "NGAM_NU" or np.count_nonzero(ref) > 0
    ctx.close()


def test_noalloc_rejects_bad_requests():
    spec = W.config_tiny(n=16, n_src=4, steps=1, seed=2, name="T16s")
    ctx = rt.RTContext([W.make_inputs(spec)], [1], outputs="core", ray_capacity=1 << 18)
    ctx.setup()
    ctx.step()
    ncell = spec.n ** 3
    # beyond the scratch size: refused with a message, nothing written
    big = _abi.NOALLOC_MAX_CELLS + 1
    out = np.full(4, 7.0, np.float32)
    st = ctx.L.frt_get_sparse_field_noalloc(ctx.h, 0, _abi.FIELD_ID["GAMMA_H1_TOT"], 0, 0, big, out.ctypes.data)
    assert st == _abi.FRT_ERR_INVALID
    assert (out == 7.0).all()
    st, _ = _noalloc(ctx, 0, "GAMMA_H1_TOT", 0, ncell - 10, 11)       # window past the box
    assert st == _abi.FRT_ERR_INVALID
    st, _ = _noalloc(ctx, 0, "TEMP", 0, 0, 10)                        # not a lit-cell field
    assert st == _abi.FRT_ERR_INVALID
    st, _ = _noalloc(ctx, 0, "NGAM_NU", 9, 0, 10)                     # bin out of range
    assert st == _abi.FRT_ERR_INVALID
    for f in ("GAMMA_H1_NU", "NGAM_NU"):                               # per-bin fields not kept
        st, _ = _noalloc(ctx, 0, f, 0, 0, 10)
        assert st == _abi.FRT_ERR_STATE
    st, got = _noalloc(ctx, 0, "GAMMA_H1_TOT", 0, 0, ncell)
    assert st == _abi.FRT_OK
    np.testing.assert_array_equal(got, ctx.get_field(0, "GAMMA_H1_TOT"))
    ctx.close()
