"""The hydro snapshot switch on the device (frt_update_hydro_step) against the oracle, whose
restatement is pinned bit for bit on the reference's own update_hydro_step
(tests/test_hydro_oracle.py, tests/golden/T16H.npz): T16 with the expansion after every step and
two snapshot switches with rays in flight (the second brings d(delta)/dt into the temperature
equation), every step at the contract tolerances of tests/test_gpu_parity.py, ledger included."""
import os
import sys

import numpy as np
import pytest

import parity_tools as PT
from flexrt_imaging_reion_b200 import rt, workloads as W
from oracle import oracle as O
from test_gpu_parity import check
from test_hydro_oracle import G, run_switches

pytestmark = pytest.mark.gpu


class _Recorder:
    """Runs the oracle through the T16H sequence, keeping its state after every step."""

    def __init__(self):
        self.o = O.Oracle(W.make_inputs(W.config_tiny()), int(G["seed"]))
        import tempfile
        from oracle import frtd
        self.states = []
        self._td = tempfile.mkdtemp()
        self.frtd = frtd

    def step(self):
        self.o.step()

    def cosmo_expansion(self, a, b):
        self.o.cosmo_expansion(a, b)

    def hydro_step(self, snap, a_rt, dts, zz):
        self.o.hydro_step(snap, a_rt, dts, zz)

    def dump(self, s):
        p = os.path.join(self._td, f"s{s}.frtd")
        self.o.dump(p)
        self.states.append(self.frtd.read(p))


class _Device:
    def __init__(self, precision):
        self.c = rt.RTContext([W.make_inputs(W.config_tiny())], [int(G["seed"])], precision=precision,
                              outputs="diag", ray_capacity=1 << 20)
        self.c.setup()
        self.states = [PT.device_state(self.c, 0, True)]
        self.stats = []

    def step(self):
        self.stats.append(self.c.step())

    def cosmo_expansion(self, a, b):
        self.c.cosmo_expansion(a, b)

    def hydro_step(self, snap, a_rt, dts, zz):
        self.c.hydro_step(0, snap, a_rt, dts, zz)

    def dump(self, s):
        self.states.append(PT.device_state(self.c, 0, True))


@pytest.mark.parametrize("precision", ["strict", "mixed"])
def test_hydro_switch_matches_oracle(precision):
    ref = _Recorder()
    ref.dump(0)
    run_switches(ref, ref.dump)
    dev = _Device(precision)
    run_switches(dev, dev.dump)
    dev.c.close()
    check(dev.states, ref.states, precision == "strict", stats=dev.stats)
    # the density really changed, and d(delta)/dt entered after the second switch
    assert float(G["hydro"][1][0]) == 4.0
    assert not np.array_equal(ref.states[1]["nH"], ref.states[-1]["nH"])
