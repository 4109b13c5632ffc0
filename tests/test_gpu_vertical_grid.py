"""Stretched and custom vertical grids (make_vertical_grid, src/domain.jl:238-280)
on the GPU path against the CPU oracle given the same Domain.dz.  The grid
enters the Monge-Ampere operator through its d2dz2! rows and the one-sided
Neumann rows; the transforms, tendency and time step are unchanged.  FP64
parity bar: 1e-12 relative L2 for one solve, 1e-10 after many steps."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRIDS = {
    "tanh": ("stretched", {"type": "tanh", "beta": 2.0}),
    "tanh_bottom": ("stretched", {"type": "tanh", "beta": 1.5, "surface_concentration": False}),
    "exponential": ("stretched", {"type": "exponential", "beta": 2.5}),
    "sinh": ("stretched", {"type": "sinh", "beta": 2.0}),
    "power": ("stretched", {"type": "power", "alpha": 1.7}),
    "custom": ("custom", None),
}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def domain(ssg, n, nz, grid):
    kind, sp = GRIDS[grid]
    if kind == "custom":
        sp = {"z_coords": np.cumsum(np.r_[0.0, np.geomspace(0.03, 0.25, nz - 1)])}
    return ssg.make_domain(n, n, nz, z_grid=kind, stretch_params=sp)


def make_pair(ssg, oracle_mod, n, nz, grid, *, scheme="AB2", dt=1e-3, filter_freq=5, ma_rhs="surface",
              predictor="cubic", precision="fp64", ma_tol=1e-10):
    dom = domain(ssg, n, nz, grid)
    sch = ssg.AB2_LowStorage if scheme == "AB2" else ssg.RK3
    prob = ssg.SemiGeostrophicProblem(dom, scheme=sch, dt=dt, eps=0.01, filter_freq=filter_freq, filter_order=8,
                                      filter_strength=0.1, filter_cutoff=0.65, ma_tol=ma_tol, ma_maxiter=80,
                                      ma_rhs=ma_rhs, ma_predictor=predictor, precision=precision,
                                      enable_diagnostics=False)
    orc = oracle_mod.Oracle(n, n, nz, eps=0.01, dt=dt, scheme=0 if scheme == "AB2" else 1, filter_freq=filter_freq,
                            filter_order=8, filter_strength=0.1, filter_cutoff=0.65, ma_tol=ma_tol, ma_maxiter=80,
                            ma_rhs_mode=0 if ma_rhs == "surface" else 1,
                            ma_predictor={"previous": 0, "extrapolate": 1, "quadratic": 2, "cubic": 3}[predictor],
                            dz=dom.dz)
    return dom, prob, orc


@pytest.mark.parametrize("grid", list(GRIDS))
def test_set_b_parity(require_gpu, ssg, oracle_mod, grid):
    n, nz = 64, 12
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz, grid)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 5, seed=300)
    it_g, conv_g, _ = ssg.set_b_(prob, b0, dom)
    conv_o, it_o, _ = orc.set_b(b0)
    assert conv_g and conv_o and it_g == it_o
    assert rel(prob.fields.phi, orc.get(oracle_mod.FIELD_PHI)) < 1e-12
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-12
    assert rel(prob.fields.u, orc.get(oracle_mod.FIELD_U_S)) < 1e-12
    prob.close()
    orc.close()


def test_grid_changes_the_solution(require_gpu, ssg):
    """The spacing vector reaches the device: a stretched grid's surface
    potential differs from the uniform grid's."""
    n, nz = 32, 10
    b0 = ssg.jfm_spectral_buoyancy(n, n, 4, seed=301)
    out = []
    for grid in (None, "power"):
        dom = ssg.make_domain(n, n, nz) if grid is None else domain(ssg, n, nz, grid)
        p = ssg.SemiGeostrophicProblem(dom, dt=1e-3, enable_diagnostics=False)
        ssg.set_b_(p, b0, dom)
        out.append(p.fields.phis)
        p.close()
    assert rel(out[1], out[0]) > 1e-3


@pytest.mark.parametrize("grid,scheme,nsteps,ma_rhs", [("tanh", "AB2", 30, "surface"), ("exponential", "RK3", 12, "surface"),
                                                       ("custom", "AB2", 30, "volume"), ("sinh", "RK3", 10, "volume")])
def test_many_steps_parity(require_gpu, ssg, oracle_mod, grid, scheme, nsteps, ma_rhs):
    n, nz = 64, 12
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz, grid, scheme=scheme, dt=2e-3, ma_rhs=ma_rhs)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 5, seed=310)
    ssg.set_b_(prob, b0, dom)
    orc.set_b(b0)
    st = ssg.stepforward_(prob, nsteps)
    orc.step(nsteps)
    assert st.ma_unconverged == 0
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-10
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-10
    assert rel(prob.fields.phi, orc.get(oracle_mod.FIELD_PHI)) < 1e-10
    prob.close()
    orc.close()


def test_mixed_precision_on_a_stretched_grid(require_gpu, ssg, oracle_mod):
    """FP32 transforms with FP64 solve on the tanh grid stay within 1e-6 of the
    FP64 oracle after 100 steps."""
    n, nz = 64, 12
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz, "tanh", precision="mixed", predictor="quadratic")
    b0 = ssg.jfm_spectral_buoyancy(n, n, 5, seed=320)
    ssg.set_b_(prob, b0, dom)
    orc.set_b(b0)
    ssg.stepforward_(prob, 100)
    orc.step(100)
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-6
    prob.close()
    orc.close()


def test_checkpoint_keeps_the_grid(require_gpu, ssg, tmp_path):
    n, nz = 32, 10
    for grid in ("tanh", "custom"):
        dom = domain(ssg, n, nz, grid)
        prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.RK3, dt=1e-3, enable_diagnostics=False)
        ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 4, seed=330), dom)
        ssg.stepforward_(prob, 5)
        f = ssg.save_simulation_state_full(str(tmp_path / f"state_{grid}.npz"), prob)
        ssg.stepforward_(prob, 6)
        b_ref = prob.fields.bs
        prob.close()
        prob2 = ssg.load_simulation_state_full(f)
        dom2 = prob2.domain
        assert dom2.z_grid == dom.z_grid and np.array_equal(dom2.dz, dom.dz)
        ssg.stepforward_(prob2, 6)
        assert np.array_equal(prob2.fields.bs, b_ref)
        prob2.close()


def test_gradient_on_a_stretched_grid(require_gpu, ssg):
    """Discrete adjoint on the tanh grid against central differences (1e-6)."""
    n, nz, k0, h = 32, 10, 4, 1e-6
    dom = domain(ssg, n, nz, "tanh")
    prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.RK3, dt=1e-3, filter_freq=3, filter_order=8, ma_tol=1e-13,
                                      ma_maxiter=200, enable_diagnostics=False)
    b0 = ssg.jfm_spectral_buoyancy(n, n, k0, seed=340)
    target = ssg.jfm_spectral_buoyancy(n, n, k0, seed=341)
    _, g = ssg.adjoint.misfit_loss_and_gradient(prob, b0, target, 8, 3)
    for s in (342, 343):
        d = ssg.jfm_spectral_buoyancy(n, n, k0, seed=s)
        fd = (ssg.adjoint.misfit_loss(prob, b0 + h * d, target, 8) -
              ssg.adjoint.misfit_loss(prob, b0 - h * d, target, 8)) / (2 * h)
        assert abs(float(np.sum(g * d)) - fd) / abs(fd) < 1e-6
    prob.close()


def test_setter_rejects_bad_spacings(require_gpu, ssg):
    L = ssg._lib.load()
    dom = ssg.make_domain(32, 32, 8)
    p = ssg.SemiGeostrophicProblem(dom, enable_diagnostics=False)
    dp = ctypes.POINTER(ctypes.c_double)
    for dz, n in ((np.full(7, 0.1), 7), (np.r_[0.1, 0.0, np.full(6, 0.1)], 8), (np.r_[0.1, -0.1, np.full(6, 0.1)], 8),
                  (np.r_[np.nan, np.full(7, 0.1)], 8)):
        dz = np.ascontiguousarray(dz)
        assert L.ssg_set_vertical_grid(p._ctx.h, dz.ctypes.data_as(dp), n) == ssg._lib.SSG_ERR_ARG
    p.close()


# ---- the reference's multigrid on a custom grid -------------------------------------------------------------

def mg_pair(ssg, oracle_mod, n, nz, z, n_levels, seed):
    dom = ssg.make_domain(n, n, nz, z_grid="custom", stretch_params={"z_coords": z})
    g = ssg.SSGMultigrid(dom, n_levels)
    o = oracle_mod.OracleMG(n, n, nz, n_levels=n_levels, dz=dom.dz)
    rng = np.random.default_rng(seed)
    phi = np.asfortranarray(rng.standard_normal((n, n, nz)))
    b = np.asfortranarray(np.repeat(ssg.jfm_spectral_buoyancy(n, n, 4, seed=seed + 1)[:, :, None], nz, axis=2))
    for k, v in (("phi", phi), ("b", b)):
        g.set(0, k, v)
    o.set(0, oracle_mod.MG_PHI, phi)
    o.set(0, oracle_mod.MG_RHS, b)
    return g, o


# mild (max spacing ratio < 2), moderate (< 5) and strong (> 5) stretching: the
# adaptive smoother takes a different branch for each
Z_MILD = np.cumsum(np.r_[0.0, np.geomspace(0.1, 0.18, 7)])
Z_MODERATE = np.cumsum(np.r_[0.0, 0.05, 0.2, 0.2, 0.2, 0.2, 0.2, 0.2])
Z_STRONG = np.cumsum(np.r_[0.0, 0.01, 0.01, 0.1, 0.1, 0.2, 0.2, 0.38])


@pytest.mark.parametrize("z", [Z_MILD, Z_MODERATE, Z_STRONG], ids=["mild", "moderate", "strong"])
@pytest.mark.parametrize("smoother", ["sor", "enhanced", "adaptive"])
def test_multigrid_smoothers_on_custom_grids(require_gpu, ssg, oracle_mod, z, smoother):
    g, o = mg_pair(ssg, oracle_mod, 32, 8, z, 1, 50)
    g.smooth(0, smoother, 2, 0.8, 0.1)
    o.smooth(0, {"sor": 1, "enhanced": 2, "adaptive": 3}[smoother], 2, 0.8, 0.1)
    assert rel(g.get(0, "phi"), o.get(0, oracle_mod.MG_PHI)) < 1e-11
    g.residual(0, 0.1)
    o.residual(0, 0.1)
    assert rel(g.get(0, "r"), o.get(0, oracle_mod.MG_RESIDUAL)) < 1e-11


@pytest.mark.parametrize("smoother", ["sor", "enhanced", "adaptive"])
def test_multigrid_v_cycle_on_a_custom_grid(require_gpu, ssg, oracle_mod, smoother):
    g, o = mg_pair(ssg, oracle_mod, 64, 8, Z_STRONG, 3, 60)
    g.v_cycle(smoother, 0.8, 0.1)
    o.v_cycle({"sor": 1, "enhanced": 2, "adaptive": 3}[smoother], 0.8, 0.1)
    assert rel(g.get(0, "phi"), o.get(0, oracle_mod.MG_PHI)) < 1e-9
