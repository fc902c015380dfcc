"""The FP64 checker of the adjoint (oracle/frt_oracle.cc, orc_adj_objective): its tangent-linear
derivative agrees with central finite differences of its own objective (h = 1e-4 relative) along
source-luminosity and cell-density directions and on single inputs."""
import numpy as np
import pytest

from flexrt_imaging_reion_b200 import workloads as W
from oracle import oracle as O

SPEC = W.config_tiny(n=24, n_src=8, steps=1, seed=17, name="A24", src_region=12)
LO, HI = [8, 8, 8], [16, 16, 16]


@pytest.fixture(scope="module")
def orc():
    inp = W.make_inputs(SPEC)
    o = O.Oracle(inp, 5)
    yield o, W.grid_sources(inp)
    o.close()


def test_objective_sees_rays(orc):
    o, _ = orc
    J, _, nlit = o.adj_objective(LO, HI)
    assert J > 0 and nlit > 0


@pytest.mark.parametrize("which", ["lum", "nh"])
def test_tangent_linear_matches_central_fd(orc, which):
    o, (ijk, lum) = orc
    rng = np.random.default_rng(3)
    h = 1e-4
    n3 = SPEC.n ** 3
    for _ in range(3):
        if which == "lum":
            v = rng.standard_normal(len(lum))
            _, jvp, _ = o.adj_objective(LO, HI, dlam=v)
            jp, _, _ = o.adj_objective(LO, HI, lam=1 + h * v)
            jm, _, _ = o.adj_objective(LO, HI, lam=1 - h * v)
        else:
            v = rng.standard_normal(n3)
            _, jvp, _ = o.adj_objective(LO, HI, dsc=v)
            jp, _, _ = o.adj_objective(LO, HI, sc=1 + h * v)
            jm, _, _ = o.adj_objective(LO, HI, sc=1 - h * v)
        fd = (jp - jm) / (2 * h)
        assert abs(jvp - fd) <= 1e-5 * abs(jvp), (jvp, fd)


def test_single_inputs(orc):
    """Unit directions: every source, and the source cells (always on a path)."""
    o, (ijk, lum) = orc
    h = 1e-4
    for s in range(len(lum)):
        e = np.zeros(len(lum))
        e[s] = 1.0
        _, jvp, _ = o.adj_objective(LO, HI, dlam=e)
        jp, _, _ = o.adj_objective(LO, HI, lam=1 + h * e)
        jm, _, _ = o.adj_objective(LO, HI, lam=1 - h * e)
        assert abs(jvp - (jp - jm) / (2 * h)) <= 1e-5 * max(abs(jvp), 1e-30)
    n = SPEC.n
    for c in ijk[:4]:
        e = np.zeros(n ** 3)
        e[(c[0] * n + c[1]) * n + c[2]] = 1.0
        _, jvp, _ = o.adj_objective(LO, HI, dsc=e)
        jp, _, _ = o.adj_objective(LO, HI, sc=1 + h * e)
        jm, _, _ = o.adj_objective(LO, HI, sc=1 - h * e)
        fd = (jp - jm) / (2 * h)
        assert abs(jvp - fd) <= 1e-5 * max(abs(jvp), abs(fd), 1e-30)
