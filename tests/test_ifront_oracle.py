"""I-front tracking in the sub-grid model (subgrid = TRUE, equilibrium = TRUE, ifront = TRUE, the
reference's own default configuration, user_inputs.h:11-15): the oracle's restatement
(frt_oracle.cc: the neutral-part photon budget of the ray pass, update_fion, set_Treion, the
front-averaged HI interpolants) on the synthetic RadHydro tables of tests/golden/subgrid_tables.py
reproduces the reference's own code compiled for one thread bit for bit, on every stored field
(the front fractions and crossing times included) and on the multiset of live rays, over 8 steps
in which fronts cross many cells part-way (tests/golden/T16F.npz).

The neutral part of a cell absorbs the rays' photons in ray order up to its atoms, so the result
depends on the order in which the rays reach a cell; with one thread the reference goes through
its ray slots in order, which is the order the rays were created in (the oracle's order).

One element is not compared: the reference's table import writes each RadHydro row at the gamma
index q + 1 (subgrid.cc:29-44), so its last write lands one float past the end of time_RH, which
the compiled reference lays out on tcross_new[0][0][0][0] (global_variables.cc:225, 272): that
element holds the table's last time (3.15e16 s) from the set-up on. The oracle keeps the array
as the algorithm defines it (0 until a front reaches the cell), and the test checks that no front
reaches cell 0, so nothing else depends on the overwritten value."""
import os
import sys
import tempfile

import numpy as np

from flexrt_imaging_reion_b200 import workloads as W
from oracle import frtd, oracle as O
from test_oracle_golden import _sorted_rays

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import subgrid_tables as ST  # noqa: E402

G = np.load(os.path.join(HERE, "golden", "T16F.npz"))
SPEC = W.config_tiny(steps=8)


def ifront_oracle():
    o = O.Oracle(W.make_inputs(SPEC), int(G["seed"]))
    o.set_subgrid(ST.reference_arrays(*G["span"]), G["consts"], ifront=True)
    return o


def test_ifront_matches_reference():
    o = ifront_oracle()
    with tempfile.TemporaryDirectory() as td:
        for s in G["steps"]:
            o.step()
            p = os.path.join(td, "x.frtd")
            o.dump(p)
            d = frtd.read(p)
            pre = f"s{s}_"
            for k in G.files:
                if not k.startswith(pre) or k[len(pre):].startswith("ray_") or k == pre + "scalars":
                    continue
                a, b = d[k[len(pre):]], G[k]
                if k == pre + "tcross_new":   # the import's spill past time_RH (module docstring)
                    assert b[0, 0] == np.float32(ST.reference_arrays(*G["span"])["time"][-1]) and a[0, 0] == 0
                    a, b = a.copy(), b.copy()
                    a[0, 0] = b[0, 0] = 0
                np.testing.assert_array_equal(a, b, err_msg=f"step {s} field {k}")
            assert G[pre + "tcross_flag"][0] == 0
            np.testing.assert_array_equal(d["scalars"][:9], G[pre + "scalars"][:9], err_msg=f"step {s} scalars")
            a = _sorted_rays({("x_" + k): v for k, v in d.items()}, "x_")
            b = _sorted_rays(G, pre)
            for k in a:
                np.testing.assert_array_equal(a[k], b[k], err_msg=f"step {s} rays {k}")
            # the order itself: the oracle's rays in creation order are the reference's slots in
            # order (the order the photon budgets are drawn in)
            for k in ("ray_cell", "ray_pixel", "ray_order", "ray_itheta"):
                np.testing.assert_array_equal(d[k], G[pre + k], err_msg=f"step {s} ray order {k}")
    o.close()
    # the fronts were tracked: cells part-way ionised, crossing times booked, rays absorbed
    f = G["s8_fion"]
    assert int(((f > 0) & (f < 1)).sum()) > 100
    assert int((G["s8_tcross_new"] > 0).sum()) > 100
