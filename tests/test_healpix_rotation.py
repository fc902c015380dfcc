"""Known-answer tests of the project's HEALPix NEST code (hp_nest.h, shared by the oracle shim and
the CUDA kernels) and of the rotation-coefficient table the product library builds."""
import ctypes as C

import numpy as np
import pytest


def _p2v(lib, order, pix):
    v = np.zeros(3)
    lib.orc_pix2vec(order, pix, v.ctypes.data)
    return v


def _v2p(lib, order, v):
    v = np.ascontiguousarray(v, np.float64)
    return lib.orc_vec2pix(order, v.ctypes.data)


def test_base_pixels(oracle_lib):
    # the 12 base pixels: z = +-2/3 in the caps at phi = pi/4 + k pi/2, z = 0 on the equator at phi = k pi/2
    for p in range(12):
        v = _p2v(oracle_lib, 0, p)
        assert abs(np.linalg.norm(v) - 1.0) < 1e-15
        if p < 4:
            assert abs(v[2] - 2.0 / 3.0) < 1e-15
            assert abs(np.arctan2(v[1], v[0]) % (2 * np.pi) - (np.pi / 4 + p * np.pi / 2)) < 1e-14
        elif p < 8:
            assert abs(v[2]) < 1e-15
            assert abs(np.arctan2(v[1], v[0]) % (2 * np.pi) - (p - 4) * np.pi / 2) < 1e-14
        else:
            assert abs(v[2] + 2.0 / 3.0) < 1e-15


@pytest.mark.parametrize("order", [0, 1, 2, 3, 5])
def test_roundtrip_and_children(oracle_lib, order):
    npix = 12 << (2 * order)
    zs = []
    for p in range(npix):
        v = _p2v(oracle_lib, order, p)
        zs.append(v[2])
        assert _v2p(oracle_lib, order, v) == p
        for c in range(4):     # NEST children 4p+c at order+1 lie inside pixel p
            assert _v2p(oracle_lib, order, _p2v(oracle_lib, order + 1, 4 * p + c)) == p
    # equal-area rings: the centre z values take 4 nside - 1 distinct values
    assert len(set(np.round(zs, 12))) == 4 * (1 << order) - 1


def test_high_order_roundtrip(oracle_lib):
    rng = np.random.default_rng(0)
    for order in (8, 10, 12):
        for p in rng.integers(0, 12 << (2 * order), 500):
            assert _v2p(oracle_lib, order, _p2v(oracle_lib, order, int(p))) == int(p)


def test_rotation_table_matches_reference_expressions(product_lib, oracle_lib):
    t = np.zeros((42875, 18), np.float32)
    assert product_lib.frt_build_rotation_table(t.ctypes.data) == 0
    rng = np.random.default_rng(1)
    for it in rng.integers(0, 42875, 3000):
        v = rng.standard_normal(3)
        v = (v / np.linalg.norm(v)).astype(np.float32).astype(np.float64)
        x, y, z = v.astype(np.float32)
        for direction, off in ((0, 0), (6, 9)):
            o = np.zeros(3)
            oracle_lib.orc_rotate(int(it), direction, v.ctypes.data, o.ctypes.data)
            m = t[it, off:off + 9]
            got = [(m[0] * x + m[1] * y) + m[2] * z, (m[3] * x + m[4] * y) + m[5] * z,
                   (m[6] * x + m[7] * y) + m[8] * z]
            assert [np.float32(a) for a in o] == got
