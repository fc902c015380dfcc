"""Restart files on the device, in the reference's formats: the device's writers against the
oracle's (pinned byte for byte on the reference's own writers by tests/test_restart_oracle.py),
and a device restart from the reference's records (tests/golden/T16R.npz) continued for 2 steps
against the oracle's restart (pinned bit for bit on the reference's restart path), with the
parity tolerances of tests/test_gpu_parity.py."""
import os

import numpy as np
import pytest

import parity_tools as PT
import restart_io as R
from flexrt_imaging_reion_b200 import rt, workloads as W
from oracle import oracle as O
from test_gpu_parity import check

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "T16R.npz"))
SPEC = W.config_tiny()
N3 = SPEC.n ** 3


def _device_after(steps, seed, precision="strict", outputs="diag"):
    ctx = rt.RTContext([W.make_inputs(SPEC)], [seed], precision=precision, outputs=outputs, ray_capacity=1 << 20)
    ctx.setup()
    for _ in range(steps):
        ctx.step()
    return ctx


def _rel(a, b, floor_frac=1e-6):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    floor = max(np.abs(b).max() * floor_frac, 1e-300)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def test_writers_match_oracle():
    ctx = _device_after(int(G["steps_before"]), int(G["base_seed"]))
    gas, rays, tre = ctx.write_restart()
    ctx.close()
    o = O.Oracle(W.make_inputs(SPEC), int(G["base_seed"]))
    for _ in range(int(G["steps_before"])):
        o.step()
    ogas, orays, otre = o.write_restart()
    o.close()
    assert len(gas) == len(ogas) and len(tre) == len(otre)
    a, b = R.parse_gas(gas, N3), R.parse_gas(ogas, N3)
    assert a["t"] == b["t"]
    for k in ("rho", "fion", "tcross", "f_He3", "treion_out"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in ("f_H1", "f_He1", "f_H2", "f_He2"):
        assert np.abs(a[k].astype(np.float64) - b[k]).max() <= 1e-4, k
    for k, tol in (("gamma_H1_tot", 1e-5), ("gamma_He1_tot", 1e-5), ("mfp", 1e-5), ("mfp_912", 1e-5),
                   ("avg_nh1", 1e-5), ("nH1", 1e-5), ("temp", 1e-4), ("heat_rate", 1e-4), ("cool_rate", 1e-4),
                   ("ngam_nu", 1e-5)):
        assert _rel(a[k], b[k]).max() <= tol, (k, _rel(a[k], b[k]).max())
    ta, tb = R.parse_treion(tre, N3), R.parse_treion(otre, N3)
    np.testing.assert_array_equal(ta["flag"], tb["flag"])
    np.testing.assert_array_equal(ta["treion"], tb["treion"])
    assert (ta["tcross_flag"] == 0).all() and (ta["neutral_flag"] == 1).all()
    ra, rb = R.parse_rays(rays), R.parse_rays(orays)
    assert len(ra) == len(rb)

    def key(r):
        return (int(r["cell"]), int(r["order"]), int(r["pixel"]), int(r["itheta"]), r["x"].tobytes(),
                r["y"].tobytes(), r["z"].tobytes(), r["r"].tobytes())

    for x, y in zip(sorted(ra, key=key), sorted(rb, key=key)):
        assert key(x) == key(y)
        assert np.abs(x["nphot"].astype(np.float64) - y["nphot"]).max() <= 1e-5 * y["nphot"].astype(np.float64).sum()


@pytest.mark.parametrize("precision", ["strict", "mixed"])
def test_restart_from_reference_records(precision):
    files = (G["gas"].tobytes(), G["tre"].tobytes(), G["rays_compact"].tobytes())
    seed = int(G["seed"])
    steps = len(G["steps"])
    inp = W.make_inputs(SPEC)
    ref = PT.oracle_restart_states(inp, seed, files, steps)
    ctx = rt.RTContext([inp], [seed], precision=precision, outputs="diag", ray_capacity=1 << 20)
    ctx.setup_restart([files])
    states = [PT.device_state(ctx, 0, True)]
    assert ctx.num_rays() == len(ref[0]["ray_order"])
    assert abs(ctx.box_scalars(0)["t"] - float(ref[0]["scalars"][0])) <= 1e-6 * float(ref[0]["scalars"][0])
    for _ in range(steps):
        ctx.step()
        states.append(PT.device_state(ctx, 0, True))
    ctx.close()
    check(states[1:], ref[1:], precision == "strict", merged=True)


def test_device_round_trip_keeps_rays():
    ctx = _device_after(3, 11, precision="mixed", outputs="core")
    gas, rays, tre = ctx.write_restart()
    n0 = ctx.num_rays()
    ctx.close()
    c2 = rt.RTContext([W.make_inputs(SPEC)], [11], ray_capacity=1 << 20)
    c2.setup_restart([(gas, tre, rays)])
    gas2, rays2, tre2 = c2.write_restart()
    dropped = int(R.parse_rays(rays)[0]["nphot"][0] == 0) if n0 else 0
    assert c2.num_rays() == n0 - dropped
    assert tre2 == tre
    keep = R.parse_rays(rays)[dropped:]
    assert R.ray_multiset(R.parse_rays(rays2)) == R.ray_multiset(keep)
    a, b = R.parse_gas(gas2, N3), R.parse_gas(gas, N3)
    for k in ("rho", "temp", "f_H1", "f_He1", "heat_rate", "cool_rate"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    c2.close()


def test_reader_rejects_malformed_records():
    c = rt.RTContext([W.make_inputs(SPEC)], [1], ray_capacity=1 << 16)
    assert c.L.frt_read_gas(c.h, 0, b"\0" * 10, 10) == 1
    gas = G["gas"].tobytes()
    assert c.L.frt_read_gas(c.h, 0, gas[:-4], len(gas) - 4) == 1
    rays = G["rays_compact"].tobytes()
    assert c.L.frt_read_rays(c.h, 0, rays[:-8], len(rays) - 8) == 1
    c.close()
