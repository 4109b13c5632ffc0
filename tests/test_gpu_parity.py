"""GPU path (libssg_b200.so through its C ABI) against the CPU oracle on the
same seeded inputs.  FP64 throughout: tolerances are relative L2 norms,
1e-12 for one operation and 1e-10 after many steps (the bar of the
plain-FP64 path)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make_pair(ssg, oracle_mod, n, nz, *, scheme="AB2", dt=1e-3, eps=0.01, filter_freq=10, filter_order=8,
              filter_strength=0.1, filter_cutoff=0.65, ma_tol=1e-10, ma_maxiter=60, ma_per_stage=True,
              ma_rhs="surface", ma_predictor="cubic"):
    dom = ssg.make_domain(n, n, nz)
    sch = ssg.AB2_LowStorage if scheme == "AB2" else ssg.RK3
    prob = ssg.SemiGeostrophicProblem(dom, scheme=sch, dt=dt, eps=eps, filter_freq=filter_freq,
                                      filter_order=filter_order, filter_strength=filter_strength,
                                      filter_cutoff=filter_cutoff, ma_tol=ma_tol, ma_maxiter=ma_maxiter,
                                      ma_per_stage=ma_per_stage, ma_rhs=ma_rhs, ma_predictor=ma_predictor,
                                      enable_diagnostics=False)
    orc = oracle_mod.Oracle(n, n, nz, eps=eps, dt=dt, scheme=0 if scheme == "AB2" else 1,
                            filter_freq=filter_freq, filter_order=filter_order, filter_strength=filter_strength,
                            filter_cutoff=filter_cutoff, ma_tol=ma_tol, ma_maxiter=ma_maxiter,
                            ma_per_stage=1 if ma_per_stage else 0, ma_rhs_mode=0 if ma_rhs == "surface" else 1,
                            ma_predictor={"previous": 0, "extrapolate": 1, "quadratic": 2, "cubic": 3}[ma_predictor])
    return dom, prob, orc


@pytest.mark.parametrize("n,nz,k0", [(32, 8, 4), (64, 8, 5), (128, 16, 6)])
def test_set_b_parity(require_gpu, ssg, oracle_mod, n, nz, k0):
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz)
    b0 = ssg.jfm_spectral_buoyancy(n, n, k0, seed=100 + n)
    it_g, conv_g, upd_g = ssg.set_b_(prob, b0, dom)
    conv_o, it_o, upd_o = orc.set_b(b0)
    assert conv_g and conv_o and it_g == it_o
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-13
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-12
    assert rel(prob.fields.phi, orc.get(oracle_mod.FIELD_PHI)) < 1e-12
    assert rel(prob.fields.u, orc.get(oracle_mod.FIELD_U_S)) < 1e-12
    assert rel(prob.fields.v, orc.get(oracle_mod.FIELD_V_S)) < 1e-12


@pytest.mark.parametrize("scheme", ["AB2", "RK3"])
def test_single_step_parity(require_gpu, ssg, oracle_mod, scheme):
    n, nz = 64, 8
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz, scheme=scheme, filter_freq=1)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 5, seed=7)
    ssg.set_b_(prob, b0, dom)
    orc.set_b(b0)
    ssg.stepforward_(prob, 1)
    orc.step(1)
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-12
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-12


@pytest.mark.parametrize("scheme,nsteps,predictor", [("AB2", 30, "extrapolate"), ("RK3", 12, "extrapolate"),
                                                     ("AB2", 30, "quadratic"), ("RK3", 12, "quadratic"),
                                                     ("AB2", 30, "cubic"), ("RK3", 12, "cubic"),
                                                     ("AB2", 10, "previous")])
def test_many_steps_parity(require_gpu, ssg, oracle_mod, scheme, nsteps, predictor):
    n, nz = 64, 8
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz, scheme=scheme, dt=2e-3, filter_freq=5, ma_predictor=predictor)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 5, seed=21)
    ssg.set_b_(prob, b0, dom)
    orc.set_b(b0)
    st = ssg.stepforward_(prob, nsteps)
    orc.step(nsteps)
    assert st.ma_unconverged == 0
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-10
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-10
    t, step = orc.time()
    assert prob.clock.step == step and abs(prob.clock.t - t) < 1e-15


def test_config1_128x16_ab2_parity(require_gpu, ssg, oracle_mod):
    """128^2 x 16, AB2 dt = 1e-3, k0 = 6, filter order 8 / cutoff 0.65 (the
    CPU-runnable configuration), 20 steps."""
    n, nz = 128, 16
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz, scheme="AB2", dt=1e-3)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 6, seed=1)
    ssg.set_b_(prob, b0, dom)
    orc.set_b(b0)
    ssg.stepforward_(prob, 20)
    orc.step(20)
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-10
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-10


@pytest.mark.parametrize("scheme", ["AB2", "RK3"])
def test_frozen_streamfunction_parity(require_gpu, ssg, oracle_mod, scheme):
    """ma_per_stage = False: phi_s solved once by set_b and then frozen, as
    the reference's time step does (src/nonlinear.jl:22-36)."""
    n, nz = 64, 8
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz, scheme=scheme, ma_per_stage=False)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 5, seed=3)
    ssg.set_b_(prob, b0, dom)
    orc.set_b(b0)
    phis0 = prob.fields.phis
    ssg.stepforward_(prob, 15)
    orc.step(15)
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-10
    assert np.array_equal(prob.fields.phis, phis0)


def test_volume_rhs_parity(require_gpu, ssg, oracle_mod):
    """ma_rhs = 'volume': b_s replicated over z as the volume right-hand side
    (src/poisson.jl:1077, 1096-1113)."""
    n, nz = 32, 8
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz, ma_rhs="volume")
    b0 = ssg.jfm_spectral_buoyancy(n, n, 4, seed=8)
    ssg.set_b_(prob, b0, dom)
    orc.set_b(b0)
    assert rel(prob.fields.phi, orc.get(oracle_mod.FIELD_PHI)) < 1e-12
    ssg.stepforward_(prob, 5)
    orc.step(5)
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-11


def test_set_get_roundtrip(require_gpu, ssg):
    """A field inside the dealiased space survives set/get exactly."""
    n, nz = 64, 8
    dom = ssg.make_domain(n, n, nz)
    prob = ssg.SemiGeostrophicProblem(dom, enable_diagnostics=False)
    b = ssg.jfm_spectral_buoyancy(n, n, 5, seed=4)
    prob.fields.bs = b
    assert np.abs(prob.fields.bs - b).max() < 1e-14 * np.abs(b).max() * n
    prob.clock.db_dt_old = 2 * b
    assert np.abs(prob.clock.db_dt_old - 2 * b).max() < 1e-14 * np.abs(b).max() * n


def test_step_until_shortens_last_step(require_gpu, ssg, oracle_mod):
    n, nz = 32, 8
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz, dt=1e-3)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 4, seed=5)
    ssg.set_b_(prob, b0, dom)
    orc.set_b(b0)
    ssg.step_until_(prob, 0.0105)
    assert prob.clock.step == 11 and prob.clock.t == 0.0105
    orc.step(10)
    orc.step(1, 0.0105 - orc.time()[0])
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-11


def test_deterministic(require_gpu, ssg):
    n, nz = 64, 8
    outs = []
    for _ in range(2):
        dom = ssg.make_domain(n, n, nz)
        prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.RK3, dt=1e-3, enable_diagnostics=False)
        ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 5, seed=6), dom)
        ssg.stepforward_(prob, 5)
        outs.append(prob.fields.bs)
        prob.close()
    assert np.array_equal(outs[0], outs[1])


def test_nonfinite_is_reported(require_gpu, ssg):
    n, nz = 32, 8
    dom = ssg.make_domain(n, n, nz)
    prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.AB2_LowStorage, dt=1e-3, ma_per_stage=False,
                                      enable_diagnostics=False)
    b = ssg.jfm_spectral_buoyancy(n, n, 4, seed=1)
    b[3, 4] = np.nan
    prob.fields.bs = b
    with pytest.raises(ssg.SsgError) as e:
        ssg.stepforward_(prob, 1)
    assert e.value.status == ssg._lib.SSG_ERR_NONFINITE


def test_not_converged_is_reported(require_gpu, ssg):
    """ma_maxiter = 1 forces the non-converged outcome (solve_ssg_equation's
    converged = false, src/poisson.jl:943-958)."""
    n, nz = 32, 8
    dom = ssg.make_domain(n, n, nz)
    prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.RK3, ma_maxiter=1, enable_diagnostics=False)
    it, conv, upd = ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 4, seed=2), dom)
    assert it == 1 and not conv and upd > 0
    st = ssg.stepforward_(prob, 2)
    assert st.ma_unconverged == st.ma_solves == 6  # three solves per RK3 step


def test_full_size_1024x32_set_b_parity(require_gpu, ssg, oracle_mod):
    """The benchmark grid (1024^2 x 32, k0 = 16): the Monge-Ampere solve of
    set_b matches the oracle (a size-independent check of the whole solve at
    full size: same iterations, same potential)."""
    n, nz = 1024, 32
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz, dt=2.5e-4)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 16, seed=2024)
    it_g, conv_g, _ = ssg.set_b_(prob, b0, dom)
    conv_o, it_o, _ = orc.set_b(b0)
    assert conv_g and conv_o and it_g == it_o
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-11


def test_full_size_properties(require_gpu, ssg):
    """At 1024^2 x 32 over 20 AB2 steps: the mean stays zero, the energy
    changes by O(dt) only, and every solve converges."""
    n, nz = 1024, 32
    dom = ssg.make_domain(n, n, nz)
    prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.AB2_LowStorage, dt=2.5e-4, filter_order=8,
                                      enable_diagnostics=False)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 16, seed=2024)
    ssg.set_b_(prob, b0, dom)
    e0 = float(np.mean(prob.fields.bs ** 2))
    st = ssg.stepforward_(prob, 20)
    b = prob.fields.bs
    assert st.ma_unconverged == 0
    assert abs(b.mean()) < 1e-12
    assert abs(float(np.mean(b ** 2)) - e0) / e0 < 1e-2


@pytest.mark.parametrize("scheme,n,nz,k0,nsteps", [("AB2", 128, 16, 6, 100), ("RK3", 64, 8, 5, 30),
                                                    ("AB2", 256, 16, 8, 40)])
def test_mixed_precision_error_bound(require_gpu, ssg, scheme, n, nz, k0, nsteps):
    """precision='mixed' (FP32 Monge-Ampere transforms, FP64 solve and
    accumulation) stays within 1e-6 relative L2 of the FP64 GPU path."""
    outs = {}
    for prec in ("fp64", "mixed"):
        dom = ssg.make_domain(n, n, nz)
        sch = ssg.AB2_LowStorage if scheme == "AB2" else ssg.RK3
        prob = ssg.SemiGeostrophicProblem(dom, scheme=sch, dt=1e-3, eps=0.01, filter_order=8, precision=prec,
                                          enable_diagnostics=False)
        ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, k0, seed=31), dom)
        st = ssg.stepforward_(prob, nsteps)
        assert st.ma_unconverged == 0
        outs[prec] = (prob.fields.bs, prob.fields.phis, st.ma_iterations)
        prob.close()
    assert rel(outs["mixed"][0], outs["fp64"][0]) < 1e-6
    assert rel(outs["mixed"][1], outs["fp64"][1]) < 1e-5


@pytest.mark.parametrize("ftype,kw", [
    (0, dict(filter_strength=2.0, filter_order=4, filter_cutoff=0.3)),
    (1, dict(filter_strength=1e-4, filter_order=2)),
    (2, dict(filter_cutoff=0.4)),
    (3, dict(filter_cutoff=0.2, filter_order=3)),
])
def test_filter_types_parity(require_gpu, ssg, oracle_mod, ftype, kw):
    """apply_spectral_filter! with each filter type of src/filter.jl."""
    n, nz = 64, 8
    objs = {0: ssg.ExponentialFilter(kw.get("filter_strength", 1.0), kw.get("filter_order", 4), kw.get("filter_cutoff", 0.65)),
            1: ssg.HyperviscosityFilter(kw.get("filter_strength", 0.0), kw.get("filter_order", 2)),
            2: ssg.CutoffFilter(kw.get("filter_cutoff", 0.65)),
            3: ssg.CesaroFilter(kw.get("filter_cutoff", 0.5), kw.get("filter_order", 2))}
    dom = ssg.make_domain(n, n, nz)
    prob = ssg.SemiGeostrophicProblem(dom, dt=1e-2, filter=objs[ftype], enable_diagnostics=False)
    orc = oracle_mod.Oracle(n, n, nz, dt=1e-2, filter_type=ftype, **kw)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 12, seed=17)
    ssg.set_b_(prob, b0, dom)
    orc.set_b(b0)
    b = prob.fields.bs
    ssg.apply_spectral_filter_(prob)
    assert rel(prob.fields.bs, orc.filter(b)) < 1e-13
    # the same transfer function installed as a custom table gives the same result
    prob.fields.bs = b
    tab_fn = {0: ssg.exponential_transfer, 2: ssg.cutoff_transfer, 3: ssg.cesaro_transfer}
    if ftype in tab_fn:
        f = objs[ftype]
        custom = ssg.CustomFilter(lambda kn, kx, ky, fn=tab_fn[ftype], f=f: fn(kn, f))
        ssg.apply_spectral_filter_(prob, dom, custom)
        assert rel(prob.fields.bs, orc.filter(b)) < 1e-13


def test_diagnostics_match_fields(require_gpu, ssg, oracle_mod):
    """Device diagnostics equal the integrals of the host-side fields."""
    n, nz = 64, 8
    dom, prob, orc = make_pair(ssg, oracle_mod, n, nz)
    ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 5, seed=23), dom)
    ssg.stepforward_(prob, 3)
    d = ssg.diagnostics(prob)
    u, v, b = prob.fields.u, prob.fields.v, prob.fields.bs
    area = dom.Lx * dom.Ly
    assert d["kinetic_energy"] == pytest.approx(0.5 * np.mean(u * u + v * v) * area, rel=1e-12)
    assert d["buoyancy_variance"] == pytest.approx(np.mean(b * b) * area, rel=1e-12)
    assert abs(d["total_buoyancy"]) < 1e-12
    assert d["step"] == 3 and d["ma_last_iterations"] > 0


@pytest.mark.parametrize("scheme", ["AB2", "RK3"])
@pytest.mark.parametrize("predictor", ["extrapolate", "quadratic", "cubic"])
def test_checkpoint_restore_continues_bit_for_bit(require_gpu, ssg, tmp_path, scheme, predictor):
    n, nz = 64, 8
    dom = ssg.make_domain(n, n, nz)
    sch = ssg.AB2_LowStorage if scheme == "AB2" else ssg.RK3
    prob = ssg.SemiGeostrophicProblem(dom, scheme=sch, dt=1e-3, filter_freq=4, ma_predictor=predictor,
                                      enable_diagnostics=False)
    ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 5, seed=29), dom)
    ssg.stepforward_(prob, 7)
    f = ssg.save_simulation_state_full(str(tmp_path / "state.npz"), prob)
    ssg.stepforward_(prob, 9)
    b_ref, t_ref, s_ref = prob.fields.bs, prob.clock.t, prob.clock.step
    prob.close()
    prob2 = ssg.load_simulation_state_full(f, dom)
    assert prob2.clock.step == 7
    ssg.stepforward_(prob2, 9)
    assert np.array_equal(prob2.fields.bs, b_ref)
    assert prob2.clock.t == t_ref and prob2.clock.step == s_ref
    # a checkpoint of another grid is rejected
    other = ssg.SemiGeostrophicProblem(ssg.make_domain(32, 32, nz), enable_diagnostics=False)
    blob = np.load(f)["ssg_b200/state"]
    rc = ssg._lib.load().ssg_restore(other._ctx.h, blob.ctypes.data, blob.size)
    assert rc == ssg._lib.SSG_ERR_ARG
    with pytest.raises(ValueError, match="Grid incompatibility"):
        ssg.load_simulation_state_full(f, ssg.make_domain(32, 32, nz))


def _filter_objects(ssg):
    return {
        "exponential": ssg.ExponentialFilter(0.5, 6, 0.6),
        "hyperviscosity": ssg.HyperviscosityFilter(1e-6, 2),
        "cutoff": ssg.CutoffFilter(0.55),
        "cesaro": ssg.CesaroFilter(0.4, 3),
        "custom": ssg.CustomFilter(lambda kn, kx, ky, a=2.0: 1.0 / (1.0 + a * kn ** 8)),
    }


@pytest.mark.parametrize("ftype", ["exponential", "hyperviscosity", "cutoff", "cesaro", "custom"])
def test_checkpoint_keeps_the_filter(require_gpu, ssg, tmp_path, ftype):
    """A restored problem filters with the saved filter: every filter type,
    a custom transfer table included, continues bit for bit."""
    n, nz = 64, 8
    dom = ssg.make_domain(n, n, nz)
    prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.AB2_LowStorage, dt=1e-3, filter_freq=2,
                                      filter=_filter_objects(ssg)[ftype], enable_diagnostics=False)
    ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 12, seed=41), dom)
    ssg.stepforward_(prob, 3)
    f = ssg.save_simulation_state_full(str(tmp_path / "s.npz"), prob)
    ssg.stepforward_(prob, 6)
    b_ref = prob.fields.bs
    prob.close()
    prob2 = ssg.load_simulation_state_full(f)
    ssg.stepforward_(prob2, 6)
    assert np.array_equal(prob2.fields.bs, b_ref)
    prob2.close()


def test_checkpoint_named_datasets(require_gpu, ssg, oracle_mod, tmp_path):
    """The file carries the reference's datasets under its key paths, with
    the values of the live problem; a file holding only those datasets (as
    one the reference wrote) loads, and the run continues from it to the
    parity tolerance of a re-solved potential."""
    n, nz = 64, 8
    dom = ssg.make_domain(n, n, nz)
    prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.AB2_LowStorage, dt=1e-3, filter_freq=5, filter_strength=0.1,
                                      enable_diagnostics=True)
    ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 5, seed=43), dom)
    ssg.stepforward_(prob, 12)
    f = ssg.save_simulation_state_full(str(tmp_path / "s.npz"), prob)
    z = np.load(f)
    assert float(z["time"]) == prob.clock.t and int(z["step"]) == 12 and float(z["dt"]) == 1e-3
    assert (int(z["grid/Nx"]), int(z["grid/Ny"]), int(z["grid/Nz"])) == (n, n, nz)
    assert np.array_equal(z["grid/kx"], dom.kx) and np.array_equal(z["grid/dz"], dom.dz)
    assert np.array_equal(z["fields/surface/buoyancy"], prob.fields.bs)
    assert np.array_equal(z["fields/surface/streamfunction"], prob.fields.phis)
    assert np.array_equal(z["fields/3d/streamfunction"], prob.fields.phi)
    assert rel(z["fields/3d/u_velocity"][:, :, -1], prob.fields.u) < 1e-12
    assert rel(z["fields/3d/v_velocity"][:, :, -1], prob.fields.v) < 1e-12
    bh = z["fields/spectral/2d/buoyancy_real"] + 1j * z["fields/spectral/2d/buoyancy_imag"]
    assert bh.shape == (n, n // 2 + 1) and rel(np.fft.irfft2(bh, s=(n, n), axes=(0, 1)), prob.fields.bs) < 1e-14
    assert z["fields/spectral/3d/streamfunction_real"].shape == (n, n // 2 + 1, nz)
    assert str(z["timestepper/scheme"]) == "AB2_LowStorage" and int(z["timestepper/filter_freq"]) == 5
    assert np.array_equal(z["timestepper/db_dt_old"], prob.clock.db_dt_old)
    assert len(z["diagnostics/times"]) > 0 and str(z["metadata/file_type"]) == "complete_simulation_state"
    # the reference's datasets alone
    named = {k: z[k] for k in z.files if not k.startswith("ssg_b200/")}
    g = str(tmp_path / "named.npz")
    np.savez(g, **named)
    ssg.stepforward_(prob, 8)
    b_ref = prob.fields.bs
    prob.close()
    prob2 = ssg.load_simulation_state_full(g, dom)
    assert prob2.clock.step == 12 and prob2.clock.t == float(z["time"])
    assert rel(prob2.fields.phis, z["fields/surface/streamfunction"]) < 1e-10
    ssg.stepforward_(prob2, 8)
    assert rel(prob2.fields.bs, b_ref) < 1e-9
    prob2.close()


@pytest.mark.parametrize("scheme,precision", [("AB2", "fp64"), ("AB2", "mixed"), ("RK3", "fp64")])
def test_short_calls_equal_one_long_call(require_gpu, ssg, scheme, precision):
    """Steps issued one call at a time (or in calls shorter than the predictor
    ring's period) replay per-phase CUDA graphs that carry the ring's buffer
    assignment forward; the result equals one call over all the steps."""
    n, nz, total = 64, 8, 13
    outs = []
    for chunks in ([total], [1] * total, [2, 3, 1, 3, 2, 2]):
        dom = ssg.make_domain(n, n, nz)
        sch = ssg.AB2_LowStorage if scheme == "AB2" else ssg.RK3
        prob = ssg.SemiGeostrophicProblem(dom, scheme=sch, dt=1e-3, filter_freq=4, filter_order=8,
                                          precision=precision, enable_diagnostics=False)
        ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 5, seed=91), dom)
        for c in chunks:
            ssg.stepforward_(prob, c)
        outs.append((prob.fields.bs, prob.fields.phi, prob.clock.t, prob.clock.step))
        # the state keeps stepping alike afterwards
        ssg.stepforward_(prob, 5)
        outs[-1] += (prob.fields.bs,)
        prob.close()
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0]) and np.array_equal(o[1], outs[0][1])
        assert o[2] == outs[0][2] and o[3] == outs[0][3]
        assert np.array_equal(o[4], outs[0][4])


@pytest.mark.parametrize("per_stage", [True, False])
def test_ab2_literal_alias_parity(require_gpu, ssg, oracle_mod, per_stage):
    """ab2_literal_alias: the AB2 tendency SSG.jl computes as written
    (fields.tmp2 is the Jacobian's output and its scratch at once,
    src/timestep.jl:159, src/transforms.jl:446,459-462), GPU against the
    oracle's literal jacobian_2d! with the aliased arrays."""
    n, nz = 64, 8
    dom = ssg.make_domain(n, n, nz)
    prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.AB2_LowStorage, dt=2e-3, filter_freq=5, filter_order=8,
                                      ma_per_stage=per_stage, ab2_literal_alias=True, enable_diagnostics=False)
    orc = oracle_mod.Oracle(n, n, nz, dt=2e-3, scheme=0, filter_freq=5, filter_order=8,
                            ma_per_stage=1 if per_stage else 0, ab2_literal_alias=1)
    plain = oracle_mod.Oracle(n, n, nz, dt=2e-3, scheme=0, filter_freq=5, filter_order=8,
                              ma_per_stage=1 if per_stage else 0)
    b0 = ssg.jfm_spectral_buoyancy(n, n, 5, seed=61)
    ssg.set_b_(prob, b0, dom)
    orc.set_b(b0)
    plain.set_b(b0)
    ssg.stepforward_(prob, 12)
    orc.step(12)
    plain.step(12)
    ref = orc.get(oracle_mod.FIELD_B_S)
    assert rel(prob.fields.bs, ref) < 1e-10
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-10
    # and it is a different tendency from the conservative Jacobian's
    assert rel(ref, plain.get(oracle_mod.FIELD_B_S)) > 1e-4
    # the adjoint covers the conservative Jacobian only
    with pytest.raises(ssg.SsgError):
        ssg.adjoint.record_(prob, b0, 2, 2)
