"""Vertical grids of make_vertical_grid (src/domain.jl:238-280 and the
stretching maps of src/domain.jl:597-729): known answers and the reference's
error behaviour.  Host-only (no device)."""
import math

import numpy as np
import pytest


def test_uniform_grid(ssg):
    z, dz = ssg.make_vertical_grid(9, 2.0)
    assert np.allclose(z, np.linspace(0, 2, 9), rtol=0, atol=1e-15)
    assert np.array_equal(dz, np.full(9, 0.25))


def test_spacing_rule_known_answer(ssg):
    """power grid, alpha = 2, Nz = 5: z = xi^2 on xi = 0, 1/4, .., 1, and
    dz = [z2 - z1, (z3 - z1)/2, (z4 - z2)/2, (z5 - z3)/2, z5 - z4] exactly."""
    z, dz = ssg.make_vertical_grid(5, 1.0, "stretched", stretch_params={"type": "power", "alpha": 2.0})
    assert np.array_equal(z, [0.0, 1 / 16, 1 / 4, 9 / 16, 1.0])
    assert np.array_equal(dz, [1 / 16, 1 / 8, 1 / 4, 3 / 8, 7 / 16])


def test_tanh_surface_concentration_runs_downwards(ssg):
    """The reference's surface-concentrated tanh map puts z = Lz at xi = 0 and
    z = 0 at xi = 1, so every spacing is negative; the bottom-concentrated map
    runs upwards.  The two are mirror images: z_surf = Lz - z_bottom."""
    Lz, nz, beta = 1.5, 12, 2.0
    zs, dzs = ssg.make_vertical_grid(nz, Lz, "stretched", stretch_params={"type": "tanh", "β": beta})
    zb, dzb = ssg.make_vertical_grid(nz, Lz, "stretched",
                                     stretch_params={"type": "tanh", "beta": beta, "surface_concentration": False})
    assert zs[0] == pytest.approx(Lz, abs=1e-15) and zs[-1] == pytest.approx(0.0, abs=1e-15)
    assert (dzs < 0).all() and (dzb > 0).all()
    assert np.allclose(zs, Lz - zb, rtol=0, atol=1e-15)
    # spacing is finest at the concentrated end
    assert abs(dzs[0]) < abs(dzs[nz // 2]) and dzb[0] < dzb[nz // 2]
    xi = np.arange(nz) / (nz - 1)
    assert np.allclose(zb, Lz * 0.5 * (1 + np.tanh(beta * (2 * xi - 1)) / math.tanh(beta)), rtol=0, atol=1e-15)


def test_exponential_and_sinh_maps(ssg):
    nz, beta = 9, 2.0
    z, dz = ssg.make_vertical_grid(nz, 1.0, "stretched", stretch_params={"type": "exponential"})
    # surface form as written: z(0) = 1 - 1/(1 - e^-2) < 0, z(1) = 1 - e^-2/(1 - e^-2)
    assert z[0] == pytest.approx(1 - 1 / (1 - math.exp(-beta)), rel=1e-15)
    assert z[-1] == pytest.approx(1 - math.exp(-beta) / (1 - math.exp(-beta)), rel=1e-15)
    assert (np.diff(dz[1:-1]) < 0).all()        # finer towards the top
    zb, _ = ssg.make_vertical_grid(nz, 1.0, "stretched",
                                   stretch_params={"type": "exponential", "surface_concentration": False})
    assert zb[0] == 0.0 and zb[-1] == pytest.approx(1.0, rel=1e-15)
    zs, dzs = ssg.make_vertical_grid(nz, 2.0, "stretched", stretch_params={"type": "sinh", "beta": 1.5})
    assert np.allclose(zs + zs[::-1], 2.0, rtol=0, atol=1e-15)   # symmetric about the middle
    assert np.allclose(dzs, dzs[::-1], rtol=0, atol=1e-15)
    assert zs[0] == pytest.approx(0.0, abs=1e-15) and zs[-1] == pytest.approx(2.0, rel=1e-15)


def test_custom_grid(ssg):
    z = np.array([0.0, 0.1, 0.3, 0.6, 1.0])
    dom = ssg.make_domain(8, 8, 5, z_grid="custom", stretch_params={"z_coords": z})
    assert np.array_equal(dom.z, z)
    assert np.allclose(dom.dz, [0.1, 0.15, 0.25, 0.35, 0.4], rtol=0, atol=1e-16)
    assert dom.z_grid == "custom"


def test_reference_errors(ssg):
    with pytest.raises(ValueError):
        ssg.make_vertical_grid(8, 1.0, "stretched")                       # no stretch_params
    with pytest.raises(ValueError):
        ssg.make_vertical_grid(8, 1.0, "custom", stretch_params={})      # no z_coords
    with pytest.raises(ValueError):
        ssg.make_vertical_grid(8, 1.0, "custom", stretch_params={"z_coords": np.arange(7.0)})
    with pytest.raises(ValueError):
        ssg.make_vertical_grid(8, 1.0, "stretched", stretch_params={"type": "cosine"})
    with pytest.raises(ValueError):
        ssg.make_vertical_grid(8, 1.0, "spiral")


def test_defaults_and_symbols(ssg):
    """type defaults to tanh with beta 2 and surface concentration; Julia's
    symbol spelling (":tanh") is accepted."""
    a = ssg.make_vertical_grid(10, 1.0, ":stretched", stretch_params={})
    b = ssg.make_vertical_grid(10, 1.0, "stretched", stretch_params={"type": ":tanh", "β": 2.0,
                                                                     "surface_concentration": True})
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    c = ssg.make_vertical_grid(10, 1.0, "stretched", stretch_params={"type": "power"})
    assert np.array_equal(c[0], 1.0 * (np.arange(10) / 9) ** 1.5)


def test_oracle_multigrid_stretched_smoothers(oracle_mod, ssg):
    """The adaptive smoother picks the enhanced smoother with metrics on a grid
    whose spacing ratio exceeds 5 (0.8 omega), and the metric rows change the
    sweep there; on a uniform grid adaptive is plain SOR."""
    n, nz = 16, 8
    z = np.cumsum(np.r_[0.0, 0.01, 0.01, 0.1, 0.1, 0.2, 0.2, 0.38])
    dom = ssg.make_domain(n, n, nz, z_grid="custom", stretch_params={"z_coords": z})
    rng = np.random.default_rng(0)
    phi = np.asfortranarray(rng.standard_normal((n, n, nz)))
    out = {}
    for sid in (1, 2, 3):
        o = oracle_mod.OracleMG(n, n, nz, n_levels=1, dz=dom.dz)
        o.set(0, oracle_mod.MG_PHI, phi)
        o.smooth(0, sid, 2, 0.8, 0.1)
        out[sid] = o.get(0, oracle_mod.MG_PHI)
    assert not np.array_equal(out[1], out[2]) and not np.array_equal(out[2], out[3])
    # adaptive = enhanced with metrics at 0.8 omega
    o = oracle_mod.OracleMG(n, n, nz, n_levels=1, dz=dom.dz)
    o.set(0, oracle_mod.MG_PHI, phi)
    o.smooth(0, 2, 2, 0.8 * 0.8, 0.1)
    assert np.array_equal(o.get(0, oracle_mod.MG_PHI), out[3])
    u = oracle_mod.OracleMG(n, n, nz, n_levels=1)
    v = oracle_mod.OracleMG(n, n, nz, n_levels=1)
    for g, sid in ((u, 1), (v, 3)):
        g.set(0, oracle_mod.MG_PHI, phi)
        g.smooth(0, sid, 2, 0.8, 0.1)
    assert np.array_equal(u.get(0, oracle_mod.MG_PHI), v.get(0, oracle_mod.MG_PHI))


def test_multigrid_rejects_coarse_levels_of_a_stretched_grid(ssg):
    """create_coarse_domain passes no stretch_params for a stretched grid, so
    the reference fails to build the coarse levels; one level is fine."""
    dom = ssg.make_domain(32, 32, 8, z_grid="stretched", stretch_params={"type": "tanh"})
    with pytest.raises(ValueError):
        ssg.SSGMultigrid(dom, n_levels=2)
