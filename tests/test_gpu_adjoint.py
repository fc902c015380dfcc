"""The adjoint of the step's Gamma field on the device (frt_adjoint) against the FP64 oracle:
objective, tangent-linear directional derivatives, and central finite differences
(h = 1e-4 relative) of the oracle's FP64 objective on 64 random inputs (32 source luminosities,
32 cell densities on the ray paths), to 1e-3 relative -- right after set-up, and after 3 steps
(rays advanced and split, attributed to their sources from their own geometry). Also: the context
state is left as it was, the call is refused once a merge has combined rays, the torch.autograd
harness, and the cost against one step."""
import numpy as np
import pytest
import torch

from flexrt_imaging_reion_b200 import rt, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SPEC = W.config_A()
SEED = 5
LO, HI = [56, 56, 56], [72, 72, 72]


@pytest.fixture(scope="module")
def setup():
    inp = W.make_inputs(SPEC)
    orc = O.Oracle(inp, SEED)
    ctx = rt.RTContext([inp], [SEED], ray_capacity=1 << 20)
    ctx.setup()
    J, dl, dnh = ctx.adjoint(LO, HI)
    nh = ctx.get_field(0, "NH").astype(np.float64)
    _, lums = W.grid_sources(inp)
    yield dict(inp=inp, orc=orc, ctx=ctx, J=J, dl=dl, dnh=dnh, nh=nh, lums=lums)
    ctx.close()
    orc.close()


def test_objective_matches_fp64_oracle(setup):
    Jo, _, nlit = setup["orc"].adj_objective(LO, HI)
    assert Jo > 0 and nlit > 100
    assert abs(setup["J"] - Jo) <= 1e-6 * Jo


def test_directional_derivatives(setup):
    """<grad, v> against the oracle's tangent-linear derivative along random directions."""
    rng = np.random.default_rng(11)
    o, lums, nh = setup["orc"], setup["lums"], setup["nh"]
    for _ in range(4):
        v = rng.standard_normal(len(lums))
        _, jvp, _ = o.adj_objective(LO, HI, dlam=v)
        dev = float(np.dot(setup["dl"] * lums, v))      # d/dlam = dJ/dL L
        assert abs(dev - jvp) <= 1e-4 * abs(jvp), (dev, jvp)
        w = rng.standard_normal(SPEC.n ** 3)
        _, jvp, _ = o.adj_objective(LO, HI, dsc=w)
        dev = float(np.dot(setup["dnh"].astype(np.float64) * nh, w))
        assert abs(dev - jvp) <= 1e-4 * abs(jvp), (dev, jvp)


def test_central_fd_on_64_inputs(setup):
    rng = np.random.default_rng(12)
    o, lums, nh, dnh = setup["orc"], setup["lums"], setup["nh"], setup["dnh"]
    n3 = SPEC.n ** 3
    h = 1e-4
    src = rng.choice(len(lums), 32, replace=False)
    cells = rng.choice(np.nonzero(dnh)[0], 32, replace=False)
    gl = setup["dl"] * lums
    gs = dnh.astype(np.float64) * nh
    scale = max(np.abs(gl).max(), np.abs(gs).max())
    bad = []
    for s in src:
        lam = np.ones(len(lums))
        lam[s] = 1 + h
        jp, _, _ = o.adj_objective(LO, HI, lam=lam)
        lam[s] = 1 - h
        jm, _, _ = o.adj_objective(LO, HI, lam=lam)
        fd = (jp - jm) / (2 * h)
        if abs(gl[s] - fd) > 1e-3 * max(abs(fd), 1e-6 * scale):
            bad.append(("L", int(s), gl[s], fd))
    for c in cells:
        sc = np.ones(n3)
        sc[c] = 1 + h
        jp, _, _ = o.adj_objective(LO, HI, sc=sc)
        sc[c] = 1 - h
        jm, _, _ = o.adj_objective(LO, HI, sc=sc)
        fd = (jp - jm) / (2 * h)
        if abs(gs[c] - fd) > 1e-3 * max(abs(fd), 1e-6 * scale):
            bad.append(("nH", int(c), gs[c], fd))
    assert not bad, bad


def test_state_untouched(setup):
    """Adjoint calls (after set-up and after a step) leave the run as it would have been."""
    inp = setup["inp"]
    with rt.RTContext([inp], [SEED], ray_capacity=1 << 20) as ref:
        ref.setup()
        ref.step()
        st_ref = ref.step()
        g_ref = ref.get_field(0, "GAMMA_H1_TOT")
        rays_ref = ref.rays(0)
    with rt.RTContext([inp], [SEED], ray_capacity=1 << 20) as c:
        c.setup()
        c.adjoint(LO, HI)
        c.step()
        c.adjoint(LO, HI)
        c.adjoint(LO, HI)
        st = c.step()
        # the ray tree is deterministic; Gamma sums are float atomics in any order (1e-6)
        assert st["crossings"] == st_ref["crossings"] and st["rays_alive"] == st_ref["rays_alive"]
        r = c.rays(0)
        assert sorted(zip(r["ray_cell"].tolist(), r["ray_pixel"].tolist())) == \
            sorted(zip(rays_ref["ray_cell"].tolist(), rays_ref["ray_pixel"].tolist()))
        np.testing.assert_allclose(c.get_field(0, "GAMMA_H1_TOT"), g_ref, rtol=1e-5, atol=0)


def test_refused_after_merge():
    """A merge combines rays of several sources (ray_tracing.cc:324-477): no per-source
    derivative exists after it."""
    spec = W.config_tiny(n=16, n_src=10, steps=8, seed=9, name="T16N", ray_per_cell_max=13, lum_min=1e53,
                         lum_max=1e55)
    with rt.RTContext([W.make_inputs(spec)], [4], ray_capacity=1 << 20) as c:
        c.setup()
        merged = 0
        for _ in range(spec.steps):
            merged += c.step()["rays_merged"]
            if merged:
                break
        assert merged > 0
        with pytest.raises(rt.FrtError, match="status 5"):
            c.adjoint([4, 4, 4], [12, 12, 12])


LATER_STEPS = 3


@pytest.fixture(scope="module")
def later():
    """The adjoint box after 3 steps, on the device (strict precision: its state follows the
    oracle's to ~1e-6, so the comparison measures the adjoint, not the state) and in the oracle."""
    inp = W.make_inputs(SPEC)
    orc = O.Oracle(inp, SEED)
    for _ in range(LATER_STEPS):
        orc.step()
    ctx = rt.RTContext([inp], [SEED], precision="strict", ray_capacity=1 << 20)
    ctx.setup()
    for _ in range(LATER_STEPS):
        ctx.step()
    J, dl, dnh = ctx.adjoint(LO, HI)
    nh = ctx.get_field(0, "NH").astype(np.float64)
    _, lums = W.grid_sources(inp)
    yield dict(orc=orc, ctx=ctx, J=J, dl=dl, dnh=dnh, nh=nh, lums=lums)
    ctx.close()
    orc.close()


def test_later_step_objective(later):
    Jo, _, nlit = later["orc"].adj_objective(LO, HI)
    assert Jo > 0 and nlit > 100
    assert abs(later["J"] - Jo) <= 1e-5 * Jo, (later["J"], Jo)


def test_later_step_directional_derivatives(later):
    """<grad, v> against the oracle's tangent-linear derivative along random directions: every
    ray's photons are attributed to the right source (a wrong attribution moves <dL, v> by O(1))."""
    rng = np.random.default_rng(21)
    o, lums, nh = later["orc"], later["lums"], later["nh"]
    for _ in range(4):
        v = rng.standard_normal(len(lums))
        _, jvp, _ = o.adj_objective(LO, HI, dlam=v)
        dev = float(np.dot(later["dl"] * lums, v))
        assert abs(dev - jvp) <= 1e-4 * abs(jvp), (dev, jvp)
        w = rng.standard_normal(SPEC.n ** 3)
        _, jvp, _ = o.adj_objective(LO, HI, dsc=w)
        dev = float(np.dot(later["dnh"].astype(np.float64) * nh, w))
        assert abs(dev - jvp) <= 1e-4 * abs(jvp), (dev, jvp)


def test_later_step_central_fd(later):
    rng = np.random.default_rng(22)
    o, lums, nh, dnh = later["orc"], later["lums"], later["nh"], later["dnh"]
    h = 1e-4
    gl = later["dl"] * lums
    gs = dnh.astype(np.float64) * nh
    scale = max(np.abs(gl).max(), np.abs(gs).max())
    bad = []
    for s_ in rng.choice(np.nonzero(gl)[0], 16, replace=False):
        lam = np.ones(len(lums))
        lam[s_] = 1 + h
        jp, _, _ = o.adj_objective(LO, HI, lam=lam)
        lam[s_] = 1 - h
        jm, _, _ = o.adj_objective(LO, HI, lam=lam)
        fd = (jp - jm) / (2 * h)
        if abs(gl[s_] - fd) > 1e-3 * max(abs(fd), 1e-6 * scale):
            bad.append(("L", int(s_), gl[s_], fd))
    for c in rng.choice(np.nonzero(dnh)[0], 16, replace=False):
        sc = np.ones(SPEC.n ** 3)
        sc[c] = 1 + h
        jp, _, _ = o.adj_objective(LO, HI, sc=sc)
        sc[c] = 1 - h
        jm, _, _ = o.adj_objective(LO, HI, sc=sc)
        fd = (jp - jm) / (2 * h)
        if abs(gs[c] - fd) > 1e-3 * max(abs(fd), 1e-6 * scale):
            bad.append(("nH", int(c), gs[c], fd))
    assert not bad, bad


def test_torch_harness():
    from adjoint_torch import GammaSubboxObjective
    spec = W.config_tiny(n=24, n_src=8, steps=1, seed=17, name="A24", src_region=12)
    lo, hi = [8, 8, 8], [16, 16, 16]
    ns = len(W.grid_sources(W.make_inputs(spec))[1])
    lam = torch.ones(ns, dtype=torch.float64, requires_grad=True)
    sc = torch.ones(spec.n ** 3, dtype=torch.float64, requires_grad=True)
    J = GammaSubboxObjective.apply(lam, sc, spec, 3, lo, hi)
    (J * J).backward()
    o = O.Oracle(W.make_inputs(spec), 3)
    Jo, _, _ = o.adj_objective(lo, hi)
    v = np.random.default_rng(1).standard_normal(ns)
    _, jvp, _ = o.adj_objective(lo, hi, dlam=v)
    o.close()
    assert abs(float(J) - Jo) <= 1e-6 * Jo
    # d(J^2)/dlam = 2 J dJ/dlam
    assert abs(float(lam.grad.numpy() @ v) - 2 * Jo * jvp) <= 1e-4 * abs(2 * Jo * jvp)


def test_adjoint_cost_against_one_step(setup):
    inp = setup["inp"]
    with rt.RTContext([inp], [SEED], ray_capacity=1 << 20) as c:
        c.setup()
        c.adjoint(LO, HI, want_dl=False, want_dnh=False)   # buffers allocated on the first call
        t_adj = []
        for _ in range(5):
            c.adjoint(LO, HI, want_dl=False, want_dnh=False)
            t_adj.append(c.last_adjoint_ms())
    with rt.RTContext([inp], [SEED], ray_capacity=1 << 20) as c:
        c.setup()
        c.step()
        t_step = c.last_timing()[0]
    # device time of the adjoint's kernels against one forward step of the same box (target 3x)
    assert np.median(t_adj) <= 3 * t_step, (t_adj, t_step)
