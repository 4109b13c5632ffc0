"""Discrete adjoint of the time step (ssg_adjoint_record / ssg_adjoint) against
central finite differences of the GPU forward run and of the CPU oracle.

The functional is the squared misfit L = sum (b_T - target)^2 of the final
surface buoyancy; its gradient with respect to the initial buoyancy b0 is
checked along seeded directions d: <dL/db0, d> against
(L(b0 + h d) - L(b0 - h d)) / (2h) with h = 1e-6.  Agreement bar: 1e-6
relative.  The Monge-Ampere solves use ma_tol 1e-13 here, so that a solve
whose iteration count differs between the two perturbed runs moves L by far
less than the difference quotient resolves (with 1e-10 such a jump can reach
about 1e-5 of the quotient).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H = 1e-6


def make_prob(ssg, n, nz, scheme, *, dt=1e-3, filter_freq=5, ma_rhs="surface", ma_tol=1e-13):
    dom = ssg.make_domain(n, n, nz)
    sch = ssg.AB2_LowStorage if scheme == "AB2" else ssg.RK3
    prob = ssg.SemiGeostrophicProblem(dom, scheme=sch, dt=dt, eps=0.01, filter_freq=filter_freq, filter_order=8,
                                      filter_strength=0.1, filter_cutoff=0.65, ma_tol=ma_tol, ma_maxiter=200,
                                      ma_rhs=ma_rhs, enable_diagnostics=False)
    return dom, prob


def directions(ssg, n, k0, count, seed):
    """Smooth fields of the initial spectrum, plus one white-noise field (its
    unresolved part is removed by set_b's projection)."""
    out = [ssg.jfm_spectral_buoyancy(n, n, k0, seed=seed + 17 * i) for i in range(count - 1)]
    rng = np.random.default_rng(seed)
    out.append(np.asfortranarray(rng.standard_normal((n, n))))
    return out


def fd_check(ssg, prob, b0, target, nsteps, ckpt, dirs):
    L, g = ssg.adjoint.misfit_loss_and_gradient(prob, b0, target, nsteps, ckpt)
    errs = []
    for d in dirs:
        lp = ssg.adjoint.misfit_loss(prob, b0 + H * d, target, nsteps)
        lm = ssg.adjoint.misfit_loss(prob, b0 - H * d, target, nsteps)
        fd = (lp - lm) / (2 * H)
        ad = float(np.sum(g * d))
        errs.append(abs(ad - fd) / abs(fd))
    return L, g, errs


@pytest.mark.parametrize("scheme,nsteps,ckpt", [("AB2", 24, 7), ("RK3", 12, 5)])
def test_gradient_matches_central_differences(require_gpu, ssg, scheme, nsteps, ckpt):
    n, nz, k0 = 64, 8, 5
    dom, prob = make_prob(ssg, n, nz, scheme)
    b0 = ssg.jfm_spectral_buoyancy(n, n, k0, seed=31)
    target = ssg.jfm_spectral_buoyancy(n, n, k0, seed=32)
    L, g, errs = fd_check(ssg, prob, b0, target, nsteps, ckpt, directions(ssg, n, k0, 4, 900))
    assert L > 0 and np.isfinite(g).all()
    assert max(errs) < 1e-6, errs
    prob.close()


def test_gradient_volume_rhs(require_gpu, ssg):
    n, nz, k0 = 32, 8, 4
    dom, prob = make_prob(ssg, n, nz, "RK3", ma_rhs="volume")
    b0 = ssg.jfm_spectral_buoyancy(n, n, k0, seed=41)
    target = ssg.jfm_spectral_buoyancy(n, n, k0, seed=42)
    _, _, errs = fd_check(ssg, prob, b0, target, 10, 4, directions(ssg, n, k0, 3, 700))
    assert max(errs) < 1e-6, errs
    prob.close()


def test_checkpoint_interval_does_not_change_the_gradient(require_gpu, ssg):
    """Recomputation reproduces the recorded trajectory bit for bit, so the
    gradient is the same for every checkpoint interval."""
    n, nz, k0 = 64, 8, 5
    dom, prob = make_prob(ssg, n, nz, "RK3", ma_tol=1e-10)
    b0 = ssg.jfm_spectral_buoyancy(n, n, k0, seed=51)
    target = ssg.jfm_spectral_buoyancy(n, n, k0, seed=52)
    grads = []
    for ckpt in (1, 4, 9, 20):
        _, g = ssg.adjoint.misfit_loss_and_gradient(prob, b0, target, 9, ckpt)
        grads.append(g)
    for g in grads[1:]:
        assert np.array_equal(g, grads[0])
    prob.close()


def test_adjoint_leaves_the_final_state(require_gpu, ssg):
    n, nz, k0 = 32, 8, 4
    dom, prob = make_prob(ssg, n, nz, "AB2", ma_tol=1e-10)
    b0 = ssg.jfm_spectral_buoyancy(n, n, k0, seed=61)
    ssg.adjoint.record_(prob, b0, 13, 4)
    bT = prob.fields.bs
    t0 = prob._ctx.time()
    g1, st = ssg.adjoint.adjoint(prob, bT)
    assert np.array_equal(prob.fields.bs, bT) and prob._ctx.time() == t0
    assert st["checkpoints"] == 5 and st["adjoint_solves"] == 13 and st["adjoint_unconverged"] == 0
    g2, _ = ssg.adjoint.adjoint(prob, bT)
    assert np.array_equal(g1, g2)
    # linear in the cotangent
    g3, _ = ssg.adjoint.adjoint(prob, 2.5 * bT)
    assert np.allclose(g3, 2.5 * g1, rtol=1e-12, atol=1e-12 * np.abs(g1).max())
    prob.close()


def test_recomputation_counts(require_gpu, ssg):
    """The recording tapes the last segment: with ckpt_every >= nsteps the
    reverse sweep recomputes nothing; otherwise every other segment once."""
    n, nz, k0 = 32, 8, 4
    dom, prob = make_prob(ssg, n, nz, "RK3", ma_tol=1e-10)
    b0 = ssg.jfm_spectral_buoyancy(n, n, k0, seed=81)
    rec = ssg.adjoint.record_(prob, b0, 6, 6)
    _, st = ssg.adjoint.adjoint(prob, b0)
    assert st["forward_solves"] == 0 and st["adjoint_solves"] == 18
    rec = ssg.adjoint.record_(prob, b0, 6, 2)
    _, st = ssg.adjoint.adjoint(prob, b0)
    assert st["forward_solves"] == 12 and rec["forward_solves"] == 19
    # a second reverse sweep of the same recording recomputes every segment
    _, st = ssg.adjoint.adjoint(prob, b0)
    assert st["forward_solves"] == 18
    prob.close()


def test_rejects_unsupported_configurations(require_gpu, ssg):
    n = 32
    dom = ssg.make_domain(n, n, 8)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 4, seed=1)
    p = ssg.SemiGeostrophicProblem(dom, scheme=ssg.RK3, dt=1e-3, precision="mixed", enable_diagnostics=False)
    with pytest.raises(ssg.SsgError):
        ssg.adjoint.record_(p, b0, 2, 1)
    p.close()
    p = ssg.SemiGeostrophicProblem(dom, scheme=ssg.RK3, dt=1e-3, ma_per_stage=False, enable_diagnostics=False)
    with pytest.raises(ssg.SsgError):
        ssg.adjoint.record_(p, b0, 2, 1)
    with pytest.raises(ssg.SsgError):
        ssg.adjoint.adjoint(p, b0)
    p.close()


def test_gradient_against_oracle_directional_derivatives(require_gpu, ssg, oracle_mod):
    """<dL/db0, d> from the GPU adjoint against central differences of the CPU
    oracle's own forward runs (the CPU restatement of the reference step)."""
    n, nz, k0, nsteps = 32, 8, 4, 8
    dom, prob = make_prob(ssg, n, nz, "RK3", filter_freq=3)
    b0 = ssg.jfm_spectral_buoyancy(n, n, k0, seed=71)
    target = ssg.jfm_spectral_buoyancy(n, n, k0, seed=72)
    _, g = ssg.adjoint.misfit_loss_and_gradient(prob, b0, target, nsteps, 3)
    prob.close()

    def oracle_loss(b):
        o = oracle_mod.Oracle(n, n, nz, eps=0.01, dt=1e-3, scheme=1, filter_freq=3, filter_order=8,
                              filter_strength=0.1, filter_cutoff=0.65, ma_tol=1e-13, ma_maxiter=200)
        o.set_b(b)
        o.step(nsteps)
        r = o.get(oracle_mod.FIELD_B_S) - target
        o.close()
        return float(np.sum(r * r))

    for d in directions(ssg, n, k0, 3, 800):
        fd = (oracle_loss(b0 + H * d) - oracle_loss(b0 - H * d)) / (2 * H)
        ad = float(np.sum(g * d))
        assert abs(ad - fd) / abs(fd) < 1e-6, (ad, fd)


def test_config4_256x16_rk3_200_steps(require_gpu, ssg):
    """The adjoint workload at full size: 256^2 x 16, spectral peak k = 8, RK3,
    dt 1e-3, 200 steps, checkpoint every 20, misfit against a second seeded
    field; central differences along 16 seeded directions."""
    n, nz, k0 = 256, 16, 8
    dom, prob = make_prob(ssg, n, nz, "RK3", filter_freq=10)
    b0 = ssg.jfm_spectral_buoyancy(n, n, k0, seed=2024)
    target = ssg.jfm_spectral_buoyancy(n, n, k0, seed=2025)
    _, _, errs = fd_check(ssg, prob, b0, target, 200, 20, directions(ssg, n, k0, 16, 4040))
    assert max(errs) < 1e-6, errs
    prob.close()
