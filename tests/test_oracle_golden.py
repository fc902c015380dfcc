"""The CPU restatement (oracle/frt_oracle.cc) against golden fixtures produced by the reference's
own C++ code compiled for one thread (tests/golden/make_golden.py): bit-exact on every stored
field and on the multiset of live rays."""
import os
import tempfile

import numpy as np
import pytest

from oracle import frtd, oracle as O
from flexrt_imaging_reion_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = {
    "T16": (W.config_tiny(), 11),
    "T16M": (W.config_tiny(n=16, n_src=6, steps=6, seed=5, name="T16M", clump_model="sqrt", ray_per_cell_max=12), 3),
    "T16N": (W.config_tiny(n=16, n_src=10, steps=8, seed=9, name="T16N", ray_per_cell_max=13, lum_min=1e53,
                           lum_max=1e55), 4),
}


def _sorted_rays(d, prefix):
    keys = np.stack([d[prefix + "ray_cell"].astype(np.int64), d[prefix + "ray_order"].astype(np.int64),
                     d[prefix + "ray_pixel"].astype(np.int64), d[prefix + "ray_itheta"].astype(np.int64)]
                    + [d[prefix + "ray_geom"][:, k].view(np.int32).astype(np.int64) for k in range(9)], axis=1)
    order = np.lexsort(keys.T[::-1])
    return {k: d[prefix + k][order] for k in ("ray_order", "ray_pixel", "ray_itheta", "ray_cell", "ray_end",
                                                "ray_geom", "ray_nphot", "ray_active")}


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_reference(name, oracle_lib):
    spec, seed = CASES[name]
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    keep = [int(s) for s in g["steps"]]
    assert int(g["seed"]) == seed
    inp = W.make_inputs(spec)
    o = O.Oracle(inp, seed)
    with tempfile.TemporaryDirectory() as td:
        for s in range(1, max(keep) + 1):
            o.step()
            if s not in keep:
                continue
            p = os.path.join(td, "x.frtd")
            o.dump(p)
            d = frtd.read(p)
            pre = f"s{s}_"
            for k in g.files:
                if not k.startswith(pre) or k[len(pre):].startswith("ray_") or k == pre + "scalars":
                    continue
                name_k = k[len(pre):]
                np.testing.assert_array_equal(d[name_k], g[k], err_msg=f"{name} step {s} field {name_k}")
            # scalars: t, dt, nphot_min, nphot_max, nphot_merge, num_thresh, total_rays, dx0, dx
            np.testing.assert_array_equal(d["scalars"][:9], g[pre + "scalars"][:9])
            a = _sorted_rays({("x_" + k): v for k, v in d.items()}, "x_")
            b = _sorted_rays(g, pre)
            for k in a:
                np.testing.assert_array_equal(a[k], b[k], err_msg=f"{name} step {s} rays {k}")
    o.close()
