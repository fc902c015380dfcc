"""Restart files in the reference's formats, pinned on the reference itself (tests/golden/T16R.npz,
written by the compiled reference): the oracle's writers reproduce the reference's restart
records after 3 steps of T16 byte for byte (rays as a multiset, slot numbers aside), and the
oracle's restart reader followed by 2 steps reproduces the reference's own restart path bit for
bit."""
import os
import tempfile

import numpy as np
import pytest

import restart_io as R
from flexrt_imaging_reion_b200 import workloads as W
from oracle import frtd, oracle as O
from test_oracle_golden import _sorted_rays

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "T16R.npz"))
SPEC = W.config_tiny()


def test_writers_match_reference_records():
    o = O.Oracle(W.make_inputs(SPEC), int(G["base_seed"]))
    for _ in range(int(G["steps_before"])):
        o.step()
    gas, rays, tre = o.write_restart()
    o.close()
    assert gas == G["gas"].tobytes()
    assert tre == G["tre"].tobytes()
    assert R.ray_multiset(R.parse_rays(rays)) == R.ray_multiset(R.parse_rays(G["rays"].tobytes()))


def test_restart_path_matches_reference():
    o = O.Oracle(W.make_inputs(SPEC), int(G["seed"]))
    o.read_restart(G["gas"].tobytes(), G["tre"].tobytes(), G["rays_compact"].tobytes())
    with tempfile.TemporaryDirectory() as td:
        for s in G["steps"]:
            o.step()
            p = os.path.join(td, f"s{s}.frtd")
            o.dump(p)
            d = frtd.read(p)
            pre = f"s{s}_"
            for k in G.files:
                if not k.startswith(pre) or k[len(pre):].startswith("ray_") or k == pre + "scalars":
                    continue
                np.testing.assert_array_equal(d[k[len(pre):]], G[k], err_msg=f"restart step {s} field {k}")
            # t, dt, nphot_min, nphot_max, nphot_merge, num_thresh; dx0, dx (total_rays counts casts)
            sc = G[pre + "scalars"]
            np.testing.assert_array_equal(d["scalars"][:6], sc[:6])
            np.testing.assert_array_equal(d["scalars"][7:9], sc[7:9])
            a = _sorted_rays({("x_" + k): v for k, v in d.items()}, "x_")
            b = _sorted_rays(G, pre)
            for k in a:
                np.testing.assert_array_equal(a[k], b[k], err_msg=f"restart step {s} rays {k}")
    o.close()


def test_reader_rejects_short_records():
    o = O.Oracle(W.make_inputs(SPEC), 1)
    with pytest.raises(ValueError):
        o.read_restart(G["gas"].tobytes()[:100], G["tre"].tobytes(), G["rays_compact"].tobytes())
    o.close()
