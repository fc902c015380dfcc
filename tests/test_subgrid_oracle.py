"""The sub-grid model (subgrid = TRUE, equilibrium = TRUE, ifront = FALSE): the oracle's
restatement (frt_oracle.cc, orc_set_subgrid) on synthetic RadHydro and overdensity tables in the
reference's own file formats (tests/golden/subgrid_tables.py) reproduces the reference's own
sub-grid code compiled for one thread bit for bit, on every stored field and on the multiset of
live rays, over 6 steps in which the ionised region grows (tests/golden/T16G.npz)."""
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

G = np.load(os.path.join(HERE, "golden", "T16G.npz"))
SPEC = W.config_tiny(steps=6)


def subgrid_oracle():
    o = O.Oracle(W.make_inputs(SPEC), int(G["seed"]))
    o.set_subgrid(ST.reference_arrays(*G["span"]), G["consts"])
    return o


def test_table_layout():
    """The gamma index q + 1 of the reference's tables runs one slot into the next row: the time
    the reference divides by in get_tradhydro_index (time_RH[Nt-1][0][0][0]) is the spill of the
    last file's row Nt - 2."""
    t = ST.reference_arrays(*G["span"])["time"]
    assert t[(((ST.NT - 1) * 3 + 0) * 3 + 0) * 3 + 0] == t[(((ST.NT - 2) * 3 + 2) * 3 + 2) * 3 + 3]
    assert t[(((ST.NT - 1) * 3 + 0) * 3 + 0) * 3 + 0] < t[(((ST.NT - 1) * 3 + 0) * 3 + 0) * 3 + 1]


def test_subgrid_matches_reference():
    o = subgrid_oracle()
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
                np.testing.assert_array_equal(d[k[len(pre):]], G[k], err_msg=f"step {s} field {k}")
            np.testing.assert_array_equal(d["scalars"][:9], G[pre + "scalars"][:9], err_msg=f"step {s} scalars")
            a = _sorted_rays({("x_" + k): v for k, v in d.items()}, "x_")
            b = _sorted_rays(G, pre)
            for k in a:
                np.testing.assert_array_equal(a[k], b[k], err_msg=f"step {s} rays {k}")
    # the sub-grid model was exercised: cells ionised, HI fractions from the tables
    assert int(G["s6_treion_flag"].sum()) > 100
    o.close()
