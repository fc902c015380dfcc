"""The hydro snapshot switch between steps (update_hydro_step, gas_funcs.cc:554-752, then
get_nphot_min_max): the oracle's restatement, fed the scale factors, snapshot intervals and
redshifts the reference used, reproduces a reference run with the expansion after every step and
two snapshot switches with rays in flight bit for bit (tests/golden/T16H.npz). The second switch
is the first with a previous snapshot, so d(delta)/dt enters the temperature equation after it."""
import os
import sys
import tempfile

import numpy as np

from flexrt_imaging_reion_b200 import workloads as W
from oracle import frtd, oracle as O
from test_oracle_golden import _sorted_rays

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
G = np.load(os.path.join(HERE, "golden", "T16H.npz"))


def run_switches(o, hook=None):
    """Steps of the T16H case on an oracle-like object: step, expansion, and the switches."""
    import make_golden as MG
    snaps = MG.hydro_snapshots(W.config_tiny())
    hy = {int(r[0]): (float(r[1]), float(r[2]), float(r[3])) for r in G["hydro"]}
    n = 0
    for s in G["steps"]:
        o.step()
        o.cosmo_expansion(float(G["a_current"][s - 1]), float(G["a_prev"][s - 1]))
        if int(s) in hy:
            a_rt, dts, zz = hy[int(s)]
            o.hydro_step(snaps[n], a_rt, dts, zz)
            n += 1
        if hook:
            hook(int(s))


def test_hydro_switch_matches_reference():
    o = O.Oracle(W.make_inputs(W.config_tiny()), int(G["seed"]))

    def check(s):
        with tempfile.TemporaryDirectory() as td:
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

    run_switches(o, check)
    o.close()
