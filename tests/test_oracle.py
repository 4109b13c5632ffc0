"""Pins the CPU oracle (oracle/ssg_oracle.cpp).

Two independent anchors:
  * numpy.fft (pocketfft) for transforms, derivatives, mask, Jacobian, tendency;
  * the known-answer tests of SSG.jl's own test scripts, restated with their
    defects corrected (test/test_filter.jl, test/test_nonlinear.jl,
    test/test_timestep.jl).
"""
import math

import numpy as np
import pytest
import scipy.linalg


def grid_xy(n):
    x = 2 * np.pi / n * np.arange(n)
    return np.meshgrid(x, x, indexing="ij")


def np_tendency(phi, b, kx, ky, mask):
    n = phi.shape[0]
    KX, KY = np.meshgrid(kx, ky, indexing="ij")
    F = lambda a: np.fft.rfft2(a, axes=(0, 1))
    I = lambda s: np.fft.irfft2(s, s=(n, n), axes=(0, 1))
    u = -I(1j * KY * F(phi))
    v = I(1j * KX * F(phi))
    J = I(1j * KX * F(u * b)) + I(1j * KY * F(v * b))
    return I(F(-J) * mask)


@pytest.mark.parametrize("n", [16, 32, 64, 24])
def test_rfft2_irfft2_match_numpy(oracle_mod, n):
    rng = np.random.default_rng(n)
    b = np.asfortranarray(rng.standard_normal((n, n)))
    s = oracle_mod.rfft2(b)
    ref = np.fft.rfft2(b, axes=(0, 1))
    assert np.abs(s - ref).max() <= 1e-13 * np.abs(ref).max()
    assert np.abs(oracle_mod.irfft2(s, n) - b).max() < 1e-14 * n


def test_irfft2_complex_to_real_convention(oracle_mod):
    """Non-Hermitian ky = 0 / ky = N/2 bins: imaginary parts of those y-bins
    are dropped after the x-transform, as numpy's irfft2 does."""
    n = 32
    rng = np.random.default_rng(3)
    s = rng.standard_normal((n, n // 2 + 1)) + 1j * rng.standard_normal((n, n // 2 + 1))
    ref = np.fft.irfft2(s, s=(n, n), axes=(0, 1))
    assert np.abs(oracle_mod.irfft2(np.asfortranarray(s), n) - ref).max() < 1e-15 * n * n


@pytest.mark.parametrize("n,kxr,kyr", [(128, (-42, 41), 42), (256, (-85, 84), 85), (512, (-170, 169), 170),
                                        (1024, (-341, 340), 341)])
def test_grid_tables_and_mask(oracle_mod, ssg, n, kxr, kyr):
    o = oracle_mod.Oracle(n, n, 4)
    kx, ky, mask = o.grid_tables()
    kx2, ky2 = ssg.ic.wavenumbers(n, n)
    assert np.array_equal(kx, kx2) and np.array_equal(ky, ky2)
    assert np.array_equal(mask, ssg.twothirds_mask(n, n // 2 + 1))
    kept_kx = np.round(kx[mask[:, 0]]).astype(int)
    kept_ky = np.round(ky[mask[0, :]]).astype(int)
    assert kept_kx.min() == kxr[0] and kept_kx.max() == kxr[1]
    assert kept_ky.min() == 0 and kept_ky.max() == kyr
    assert kx[n // 2] < 0  # fftfreq puts -N/2 at the Nyquist index


def test_jacobian_analytic(oracle_mod):
    """test/test_nonlinear.jl:14-84 with the analytic Jacobian corrected:
    J(sin x cos y, cos x sin y) = cos^2 x cos^2 y - sin^2 x sin^2 y."""
    n = 32
    X, Y = grid_xy(n)
    psi = np.sin(X) * np.cos(Y)
    b = np.cos(X) * np.sin(Y)
    o = oracle_mod.Oracle(n, n, 4)
    J = o.jacobian(psi, b)
    exact = np.cos(X) ** 2 * np.cos(Y) ** 2 - np.sin(X) ** 2 * np.sin(Y) ** 2
    assert np.abs(J - exact).max() < 1e-12
    # compute_tendency! negates and dealiases (src/nonlinear.jl:22-56)
    assert np.abs(o.tendency(psi, b) + exact).max() < 1e-12


def test_tendency_matches_numpy(oracle_mod, ssg):
    n = 64
    o = oracle_mod.Oracle(n, n, 4)
    kx, ky, mask = o.grid_tables()
    phi = ssg.jfm_spectral_buoyancy(n, n, 5, seed=11) * 0.2
    b = ssg.jfm_spectral_buoyancy(n, n, 5, seed=12)
    assert np.abs(o.tendency(phi, b) - np_tendency(phi, b, kx, ky, mask)).max() < 1e-12


def test_ab2_literal_alias_tendency(oracle_mod, ssg):
    """With ab2_literal_alias the oracle's AB2 step uses the tendency the
    reference's aliased arrays produce (src/timestep.jl:159,
    src/transforms.jl:446,459-462): -P[2 d/dy(b d(phi)/dx)].  One
    forward-Euler first step with a frozen streamfunction shows it."""
    n, nz, dt = 64, 8, 1e-3
    outs = {}
    for alias in (0, 1):
        o = oracle_mod.Oracle(n, n, nz, dt=dt, scheme=0, filter_freq=0, ma_per_stage=0, ab2_literal_alias=alias)
        o.set_b(ssg.jfm_spectral_buoyancy(n, n, 5, seed=19))
        b0, phi = o.get(oracle_mod.FIELD_B_S), o.get(oracle_mod.FIELD_PHI_S)
        o.step(1)
        outs[alias] = (b0, phi, o.get(oracle_mod.FIELD_B_S), o.grid_tables())
    b0, phi, b1, (kx, ky, mask) = outs[1]
    KX, KY = np.meshgrid(kx, ky, indexing="ij")
    F = lambda a: np.fft.rfft2(a, axes=(0, 1))
    I = lambda s: np.fft.irfft2(s, s=(n, n), axes=(0, 1))
    f_alias = I(F(-2.0 * I(1j * KY * F(I(1j * KX * F(phi)) * b0))) * mask)
    scale = np.abs(f_alias).max()
    assert np.abs((b1 - b0) / dt - f_alias).max() < 1e-9 * scale
    b0p, phip, b1p, _ = outs[0]
    assert np.abs((b1p - b0p) / dt - np_tendency(phip, b0p, kx, ky, mask)).max() < 1e-9 * scale


def test_geostrophic_velocities(oracle_mod):
    """test/test_nonlinear.jl:86-148 against the surface streamfunction:
    psi = sin 2x cos y -> u = sin 2x sin y, v = 2 cos 2x cos y."""
    n = 16
    X, Y = grid_xy(n)
    o = oracle_mod.Oracle(n, n, 4)
    o.set(oracle_mod.FIELD_PHI_S, np.sin(2 * X) * np.cos(Y))
    u = o.get(oracle_mod.FIELD_U_S)
    v = o.get(oracle_mod.FIELD_V_S)
    assert np.abs(u - np.sin(2 * X) * np.sin(Y)).max() < 1e-12
    assert np.abs(v - 2 * np.cos(2 * X) * np.cos(Y)).max() < 1e-12


def test_exponential_transfer_kats(oracle_mod):
    """test/test_filter.jl:43-74 (exponential part), exact values."""
    assert oracle_mod.exponential_transfer(0.3, 1.0, 2, 0.5) == 1.0
    t = oracle_mod.exponential_transfer(0.8, 1.0, 2, 0.5)
    assert 0.0 < t < 1.0
    assert abs(t - math.exp(-((0.8 - 0.5) / 0.5) ** 2)) < 1e-15
    assert oracle_mod.exponential_transfer(1.0, 0.1, 8, 0.65) == pytest.approx(math.exp(-0.1), rel=1e-15)


def test_filter_preserves_dc(oracle_mod):
    """test/test_filter.jl:222-259: a constant field passes the exponential
    filter with sum conserved to < 1e-14."""
    n = 32
    o = oracle_mod.Oracle(n, n, 4, filter_strength=0.5, filter_order=4, filter_cutoff=0.6)
    b = np.ones((n, n))
    f = o.filter(b)
    assert abs(f.sum() - b.sum()) / b.sum() < 1e-14


def test_filter_transfer_applied(oracle_mod, ssg):
    """Filtering multiplies each mode by exponential_transfer(|k|/k_max)."""
    n = 32
    o = oracle_mod.Oracle(n, n, 4, filter_strength=2.0, filter_order=2, filter_cutoff=0.3)
    kx, ky, mask = o.grid_tables()
    rng = np.random.default_rng(0)
    b = rng.standard_normal((n, n))
    bh = np.fft.rfft2(b, axes=(0, 1))
    bh[:, 0] = np.fft.rfft2(np.fft.irfft2(bh, s=(n, n), axes=(0, 1)), axes=(0, 1))[:, 0]
    KX, KY = np.meshgrid(kx, ky, indexing="ij")
    kmax = math.hypot(np.pi / (2 * np.pi / n), np.pi / (2 * np.pi / n))
    kn = np.sqrt(KX ** 2 + KY ** 2) / kmax
    sig = np.where(kn <= 0.3, 1.0, np.exp(-2.0 * ((kn - 0.3) / 0.7) ** 2))
    ref = np.fft.irfft2(bh * sig, s=(n, n), axes=(0, 1))
    assert np.abs(o.filter(b) - ref).max() < 1e-13


def test_buoyancy_conservation_rk3(oracle_mod):
    """test/test_nonlinear.jl:194-246: sum(b) is conserved by the conservative
    Jacobian over 10 RK3 steps (streamfunction frozen, as there)."""
    n = 32
    X, Y = grid_xy(n)
    o = oracle_mod.Oracle(n, n, 4, scheme=1, dt=1e-3, ma_per_stage=0, filter_freq=0)
    b0 = np.exp(-(X - np.pi) ** 2 / 2) * np.exp(-(Y - np.pi) ** 2 / 2)
    o.set(oracle_mod.FIELD_B_S, b0)
    o.set(oracle_mod.FIELD_PHI_S, 0.1 * np.sin(X) * np.cos(Y))
    o.step(10)
    b = o.get(oracle_mod.FIELD_B_S)
    assert abs(b.sum() - b0.sum()) / abs(b0.sum()) < 1e-12


def _linear_operator(o, oracle_mod, phi, n):
    """Matrix of the (frozen-phi, hence linear) tendency b -> -P J(phi, b)."""
    L = np.zeros((n * n, n * n))
    for m in range(n * n):
        e = np.zeros(n * n)
        e[m] = 1.0
        L[:, m] = o.tendency(phi, e.reshape((n, n), order="F")).ravel(order="F")
    return L


def test_time_integrators_order(oracle_mod, ssg):
    """test/test_timestep.jl:13-131 restated without a mock tendency: with the
    streamfunction frozen the tendency is linear, L b, and the exact discrete
    solution is expm(t L) b0.  RK3 must converge at third order, AB2 (with
    its forward-Euler first step) at second order."""
    n = 16
    X, Y = grid_xy(n)
    phi = 0.5 * np.sin(X) * np.cos(Y) + 0.3 * np.cos(2 * Y)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 2, seed=5)
    o = oracle_mod.Oracle(n, n, 4, ma_per_stage=0, filter_freq=0)
    L = _linear_operator(o, oracle_mod, phi, n)
    T = 0.2
    exact = (scipy.linalg.expm(T * L) @ b0.ravel(order="F")).reshape((n, n), order="F")
    for scheme, order in ((1, 3), (0, 2)):
        errs = []
        for nsteps in (20, 40):
            oo = oracle_mod.Oracle(n, n, 4, scheme=scheme, ma_per_stage=0, filter_freq=0, dt=T / nsteps)
            oo.set(oracle_mod.FIELD_B_S, b0)
            oo.set(oracle_mod.FIELD_PHI_S, phi)
            oo.step(nsteps)
            errs.append(np.abs(oo.get(oracle_mod.FIELD_B_S) - exact).max())
        rate = math.log2(errs[0] / errs[1])
        assert rate == pytest.approx(order, abs=0.25), (scheme, errs, rate)


def mask_ext(n):
    """2/3 mask closed under conjugation: (+N/3, 0) joins (-N/3, 0)."""
    mask = np.ones((n, n // 2 + 1), bool)
    mask[n // 3:n - n // 3, :] = False
    mask[:, (2 * (n // 2 + 1)) // 3:] = False
    mask[n // 3, 0] = True
    return mask


def _dense_linear_solution(n, nz, bs, lz=1.0, dz=None):
    """Per-mode dense solve of the eps = 0 problem (numpy), for comparison.
    With ``dz`` (Domain.dz of a stretched grid) the rows are the second
    difference with spacings dz[k-1] below and dz[k] above and the one-sided
    Neumann rows over dz[0], dz[1] (bottom) and dz[-2], dz[-3] (top)."""
    kx = 2 * np.pi * np.fft.fftfreq(n, 2 * np.pi / n)
    ky = 2 * np.pi * np.fft.rfftfreq(n, 2 * np.pi / n)
    if dz is not None:
        return _dense_linear_solution_dz(n, nz, bs, np.asarray(dz, float), kx, ky)
    h = lz / (nz - 1)
    mask = mask_ext(n)
    bsh = np.fft.rfft2(bs, axes=(0, 1)) * mask
    P = np.zeros((n, n // 2 + 1, nz), complex)
    for i in range(n):
        for j in range(n // 2 + 1):
            if not mask[i, j] or (i == 0 and j == 0):
                continue
            K2 = kx[i] ** 2 + ky[j] ** 2
            A = np.zeros((nz, nz))
            r = np.zeros(nz, complex)
            for k in range(1, nz - 1):
                A[k, k - 1] = 1 / h ** 2
                A[k, k] = -2 / h ** 2 - K2
                A[k, k + 1] = 1 / h ** 2
            A[0, :3] = [-3 / (2 * h), 4 / (2 * h), -1 / (2 * h)]
            A[-1, -3:] = [1 / (2 * h), -4 / (2 * h), 3 / (2 * h)]
            r[-1] = bsh[i, j]
            P[i, j, :] = np.linalg.solve(A, r)
    return np.fft.irfft2(P, s=(n, n), axes=(0, 1))


def _dense_linear_solution_dz(n, nz, bs, dz, kx, ky):
    mask = mask_ext(n)
    bsh = np.fft.rfft2(bs, axes=(0, 1)) * mask
    A0 = np.zeros((nz, nz))
    for k in range(1, nz - 1):
        hm, hp = dz[k - 1], dz[k]
        A0[k, k - 1] = 2 / (hm * (hm + hp))
        A0[k, k] = -2 / (hm * hp)
        A0[k, k + 1] = 2 / (hp * (hm + hp))
    h1, h2 = dz[0], dz[1]
    A0[0, :3] = [-(2 * h1 + h2) / (h1 * (h1 + h2)), (h1 + h2) / (h1 * h2), -h1 / (h2 * (h1 + h2))]
    h1, h2 = dz[-2], dz[-3]
    A0[-1, -3:] = [h1 / (h2 * (h1 + h2)), -(h1 + h2) / (h1 * h2), (2 * h1 + h2) / (h1 * (h1 + h2))]
    P = np.zeros((n, n // 2 + 1, nz), complex)
    for i in range(n):
        for j in range(n // 2 + 1):
            if not mask[i, j] or (i == 0 and j == 0):
                continue
            A = A0.copy()
            for k in range(1, nz - 1):
                A[k, k] -= kx[i] ** 2 + ky[j] ** 2
            r = np.zeros(nz, complex)
            r[-1] = bsh[i, j]
            P[i, j, :] = np.linalg.solve(A, r)
    return np.fft.irfft2(P, s=(n, n), axes=(0, 1))


def test_ma_linear_limit_matches_dense_solve(oracle_mod, ssg):
    """eps = 0: one fixed-point iteration is the exact linear solve (Thomas
    per mode with the Neumann rows of src/poisson.jl:309-364)."""
    n, nz = 32, 8
    o = oracle_mod.Oracle(n, n, nz, eps=0.0, ma_tol=1e-12, ma_maxiter=5)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 4, seed=2)
    conv, iters, upd = o.set_b(b0)
    assert conv and iters == 2
    Phi = o.get(oracle_mod.FIELD_PHI)
    ref = _dense_linear_solution(n, nz, o.get(oracle_mod.FIELD_B_S))
    assert np.abs(Phi - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("grid", [{"type": "tanh", "beta": 2.0}, {"type": "exponential", "beta": 3.0},
                                  {"type": "power", "alpha": 2.0}, "custom"])
def test_ma_linear_limit_on_stretched_grids(oracle_mod, ssg, grid):
    """eps = 0 on a stretched or custom vertical grid: the oracle's Thomas solve
    with the rows of Domain.dz equals a dense per-mode solve (the tanh grid's
    spacings are negative: it runs from z = Lz down to 0)."""
    n, nz = 32, 10
    if grid == "custom":
        z = np.cumsum(np.r_[0.0, np.geomspace(0.02, 0.3, nz - 1)])
        dom = ssg.make_domain(n, n, nz, z_grid="custom", stretch_params={"z_coords": z})
    else:
        dom = ssg.make_domain(n, n, nz, z_grid="stretched", stretch_params=grid)
    o = oracle_mod.Oracle(n, n, nz, eps=0.0, ma_tol=1e-12, ma_maxiter=5, dz=dom.dz)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 4, seed=12)
    conv, iters, upd = o.set_b(b0)
    assert conv and iters == 2
    Phi = o.get(oracle_mod.FIELD_PHI)
    ref = _dense_linear_solution(n, nz, o.get(oracle_mod.FIELD_B_S), dz=dom.dz)
    assert np.abs(Phi - ref).max() < 1e-11 * np.abs(ref).max()


def test_uniform_spacing_vector_changes_nothing(oracle_mod, ssg):
    """Passing the uniform Domain.dz explicitly reproduces the default run bit
    for bit (the setter rebuilds the same rows)."""
    n, nz = 32, 8
    dom = ssg.make_domain(n, n, nz)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 4, seed=13)
    out = []
    for dz in (None, dom.dz):
        o = oracle_mod.Oracle(n, n, nz, dt=1e-3, scheme=1, dz=dz)
        o.set_b(b0)
        o.step(3)
        out.append(o.get(oracle_mod.FIELD_PHI))
        o.close()
    assert np.array_equal(out[0], out[1])


def test_ma_solution_satisfies_documented_problem(oracle_mod, ssg):
    """The converged potential satisfies the Neumann rows exactly and the
    interior equation of compute_ssg_residual! (src/poisson.jl:228-253) on the
    dealiased modes; the literal residual routine agrees."""
    n, nz, eps = 32, 8, 0.01
    o = oracle_mod.Oracle(n, n, nz, eps=eps, ma_tol=1e-13, ma_maxiter=80)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 4, seed=9)
    conv, iters, upd = o.set_b(b0)
    assert conv
    Phi = o.get(oracle_mod.FIELD_PHI)
    bs = o.get(oracle_mod.FIELD_B_S)
    h = 1.0 / (nz - 1)
    top = (3 * Phi[:, :, -1] - 4 * Phi[:, :, -2] + Phi[:, :, -3]) / (2 * h)
    bot = (-3 * Phi[:, :, 0] + 4 * Phi[:, :, 1] - Phi[:, :, 2]) / (2 * h)
    assert np.abs(top - bs).max() < 1e-10 * np.abs(bs).max()
    assert np.abs(bot).max() < 1e-10 * np.abs(bs).max()
    Phi2, r = o.ssg_residual_literal(Phi, np.zeros_like(Phi), bs, eps)
    assert np.abs(Phi2 - Phi).max() < 1e-10 * np.abs(Phi).max()  # boundary rows already hold
    rh = np.fft.rfft2(r, axes=(0, 1)) * mask_ext(n)[:, :, None]
    rh[0, 0, :] = 0
    lap_scale = np.abs(np.fft.rfft2(Phi, axes=(0, 1))).max() * (n / 3) ** 2
    assert np.abs(rh).max() < 1e-9 * lap_scale


def test_ma_nonlinear_term_is_active(oracle_mod, ssg):
    """eps > 0 changes the solution by O(eps) relative to eps = 0."""
    n, nz = 32, 8
    b0 = ssg.jfm_spectral_buoyancy(n, n, 4, seed=4)
    o0 = oracle_mod.Oracle(n, n, nz, eps=0.0)
    o1 = oracle_mod.Oracle(n, n, nz, eps=0.01)
    o0.set_b(b0)
    conv, iters, _ = o1.set_b(b0)
    assert conv and iters > 2
    p0 = o0.get(oracle_mod.FIELD_PHI_S)
    p1 = o1.get(oracle_mod.FIELD_PHI_S)
    rel = np.linalg.norm(p1 - p0) / np.linalg.norm(p0)
    assert 1e-4 < rel < 0.2
