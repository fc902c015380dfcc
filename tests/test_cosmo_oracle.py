"""The cosmological expansion between steps (update_cosmo_expansion, gas_funcs.cc:460-548): the
oracle's restatement, fed the scale factors the reference used, reproduces a reference run with
the expansion after every step bit for bit (tests/golden/T16C.npz)."""
import os
import tempfile

import numpy as np

from flexrt_imaging_reion_b200 import workloads as W
from oracle import frtd, oracle as O
from test_oracle_golden import _sorted_rays

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "T16C.npz"))


def test_expansion_matches_reference():
    o = O.Oracle(W.make_inputs(W.config_tiny()), int(G["seed"]))
    with tempfile.TemporaryDirectory() as td:
        for s in G["steps"]:
            o.step()
            o.cosmo_expansion(float(G["a_current"][s - 1]), float(G["a_prev"][s - 1]))
            p = os.path.join(td, "x.frtd")
            o.dump(p)
            d = frtd.read(p)
            pre = f"s{s}_"
            for k in G.files:
                if not k.startswith(pre) or k[len(pre):].startswith("ray_") or k == pre + "scalars":
                    continue
                np.testing.assert_array_equal(d[k[len(pre):]], G[k], err_msg=f"step {s} field {k}")
            np.testing.assert_array_equal(d["scalars"][:9], G[pre + "scalars"][:9])
            a = _sorted_rays({("x_" + k): v for k, v in d.items()}, "x_")
            b = _sorted_rays(G, pre)
            for k in a:
                np.testing.assert_array_equal(a[k], b[k], err_msg=f"step {s} rays {k}")
    o.close()
