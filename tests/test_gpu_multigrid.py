"""The reference's own multigrid functions on the GPU against their literal CPU
restatement (oracle.OracleMG).  The spectral smoother diverges within a few
sweeps and the SOR smoother ignores the right-hand side -- SSG.jl's behaviour
-- so the checks run a few sweeps from band-limited and from rough fields."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def fields(ssg, n, nz, rough, seed):
    rng = np.random.default_rng(seed)
    if rough:
        phi = rng.standard_normal((n, n, nz))
    else:
        phi = np.stack([0.1 * ssg.jfm_spectral_buoyancy(n, n, 4, seed=seed + k) for k in range(nz)], axis=2)
    b = np.repeat(ssg.jfm_spectral_buoyancy(n, n, 4, seed=seed + 99)[:, :, None], nz, axis=2)
    bs = ssg.jfm_spectral_buoyancy(n, n, 3, seed=seed + 7)
    return np.asfortranarray(phi), np.asfortranarray(b), np.asfortranarray(bs)


def pair(ssg, oracle_mod, n, nz, rough, seed, n_levels=3, bs_zero=False):
    dom = ssg.make_domain(n, n, nz)
    g = ssg.SSGMultigrid(dom, n_levels)
    o = oracle_mod.OracleMG(n, n, nz, n_levels=n_levels)
    phi, b, bs = fields(ssg, n, nz, rough, seed)
    if bs_zero:
        bs = np.zeros_like(bs)
    for lvl_obj in (g,):
        lvl_obj.set(0, "phi", phi)
        lvl_obj.set(0, "b", b)
        lvl_obj.set(0, "bs_surface", bs)
    o.set(0, oracle_mod.MG_PHI, phi)
    o.set(0, oracle_mod.MG_RHS, b)
    o.set(0, oracle_mod.MG_BS_SURFACE, bs)
    return g, o


@pytest.mark.parametrize("rough", [False, True])
def test_residual_and_boundary(require_gpu, ssg, oracle_mod, rough):
    g, o = pair(ssg, oracle_mod, 32, 8, rough, 1)
    g.residual(0, 0.1)
    o.residual(0, 0.1)
    assert rel(g.get(0, "r"), o.get(0, oracle_mod.MG_RESIDUAL)) < 1e-12
    assert rel(g.get(0, "phi"), o.get(0, oracle_mod.MG_PHI)) < 1e-13   # boundary side effect
    assert g.norm(0, "r") == pytest.approx(o.norm(0, oracle_mod.MG_RESIDUAL), rel=1e-12)


@pytest.mark.parametrize("smoother,iters", [("spectral", 1), ("spectral", 2), ("sor", 3), ("enhanced", 2),
                                            ("adaptive", 2)])
def test_smoothers(require_gpu, ssg, oracle_mod, smoother, iters):
    g, o = pair(ssg, oracle_mod, 32, 8, smoother != "spectral", 2)
    sid = {"spectral": 0, "sor": 1, "enhanced": 2, "adaptive": 3}[smoother]
    g.smooth(0, smoother, iters, 0.8, 0.1)
    o.smooth(0, sid, iters, 0.8, 0.1)
    assert rel(g.get(0, "phi"), o.get(0, oracle_mod.MG_PHI)) < 1e-11


def test_transfers(require_gpu, ssg, oracle_mod):
    g, o = pair(ssg, oracle_mod, 64, 8, True, 3)
    g.restrict(1)
    o.restrict(1)
    assert np.array_equal(g.get(1, "phi"), o.get(1, oracle_mod.MG_PHI))
    assert np.array_equal(g.get(1, "bs_surface"), o.get(1, oracle_mod.MG_BS_SURFACE))
    g.prolongate(1)
    o.prolongate(1)
    assert np.array_equal(g.get(0, "phi"), o.get(0, oracle_mod.MG_PHI))


@pytest.mark.parametrize("smoother", ["spectral", "sor"])
def test_v_cycle(require_gpu, ssg, oracle_mod, smoother):
    """One ssg_v_cycle! with bs_surface = 0, as on the reference's solve path
    (set_surface_bc_from_buoyancy! is never called there).  The spectral
    smoother may already blow up in the 50 coarsest sweeps (the preconditioner
    ignores the vertical operator); then both sides must blow up alike."""
    g, o = pair(ssg, oracle_mod, 64, 8, False, 4, bs_zero=True)
    g.v_cycle(smoother, 0.8, 0.1)
    o.v_cycle({"spectral": 0, "sor": 1}[smoother], 0.8, 0.1)
    a, b = g.get(0, "phi"), o.get(0, oracle_mod.MG_PHI)
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    if fin.all():
        assert rel(a, b) < 1e-9
    else:
        assert smoother == "spectral"


def test_coarse_levels_are_inert_on_the_reference_path(require_gpu, ssg, oracle_mod):
    """With b and bs_surface never restricted (src/poisson.jl:710-711), a
    V-cycle's coarse correction is exactly zero: the cycle's only coarse effect
    is to zero Phi at the injected points and add nothing back."""
    g, o = pair(ssg, oracle_mod, 64, 8, False, 6, bs_zero=True)
    g.restrict(1)
    g.set(1, "phi", np.zeros(g.shape(1)))
    g.smooth(1, "sor", 5, 0.8, 0.1)
    assert np.abs(g.get(1, "phi")).max() == 0.0


def test_solve_ssg_equation_reproduces_reference_behaviour(require_gpu, ssg, oracle_mod):
    """From a zero guess the SOR V-cycle leaves Phi at zero (the smoother
    ignores the right-hand side); the reported residual matches."""
    n, nz = 32, 8
    dom = ssg.make_domain(n, n, nz)
    b = np.repeat(ssg.jfm_spectral_buoyancy(n, n, 4, seed=5)[:, :, None], nz, axis=2)
    sol, diag = ssg.solve_ssg_equation(np.zeros((n, n, nz)), b, 0.1, dom, tol=1e-10, maxiter=2, smoother="sor")
    o = oracle_mod.OracleMG(n, n, nz)
    o.set(0, oracle_mod.MG_RHS, b)
    conv, it, res = o.solve(0.1, 1e-10, 2, 1, 0.8)
    assert not diag["converged"] and diag["iterations"] == it == 2
    assert diag["final_residual"] == pytest.approx(res, rel=1e-12)
    assert np.abs(sol).max() == 0.0
