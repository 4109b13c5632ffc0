"""The benchmark configurations, GPU against the CPU oracle on the same seeded
inputs (FP64), and the mixed-precision form against the FP64 GPU path.

  1: 128^2 x 16, AB2, dt 1e-3, k0 = 6, 100 steps (the CPU-runnable case)
  2: 512^2 x 32, RK3, dt 5e-4, k0 = 10 (the FP64 drop-in), 20 steps against
     the oracle -- as many as it runs in about a minute
  3: 1024^2 x 32, AB2, dt 2.5e-4, k0 = 16 (the headline grid): FP64 set_b and
     5 steps against the oracle; mixed precision against FP64 after 10, 100
     and 1000 steps, for two seeds and a sharper initial spectrum (k0 = 24)

Filter order 8, cutoff 0.65, strength 0.1 every 10 steps, eps 0.01,
ma_tol 1e-10 in every case.  Tolerances are relative L2 norms over the
surface: 1e-10 for the FP64 path, 1e-6 for mixed precision.
"""
import time

import numpy as np
import pytest

from ma_residual import ma_residual

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def pair(ssg, oracle_mod, n, nz, scheme, dt, predictor):
    dom = ssg.make_domain(n, n, nz)
    sch = ssg.AB2_LowStorage if scheme == "AB2" else ssg.RK3
    prob = ssg.SemiGeostrophicProblem(dom, scheme=sch, dt=dt, eps=0.01, filter_freq=10, filter_order=8,
                                      filter_strength=0.1, filter_cutoff=0.65, ma_tol=1e-10, ma_maxiter=60,
                                      ma_predictor=predictor, enable_diagnostics=False)
    orc = oracle_mod.Oracle(n, n, nz, eps=0.01, dt=dt, scheme=0 if scheme == "AB2" else 1, filter_freq=10,
                            filter_order=8, filter_strength=0.1, filter_cutoff=0.65, ma_tol=1e-10, ma_maxiter=60,
                            ma_predictor={"quadratic": 2, "cubic": 3}[predictor])
    return dom, prob, orc


def test_config1_full_run(require_gpu, ssg, oracle_mod):
    """Configuration 1 as specified: 100 AB2 steps."""
    n, nz = 128, 16
    dom, prob, orc = pair(ssg, oracle_mod, n, nz, "AB2", 1e-3, "cubic")
    b0 = ssg.jfm_spectral_buoyancy(n, n, 6, seed=1)
    it_g, conv_g, _ = ssg.set_b_(prob, b0, dom)
    conv_o, it_o, _ = orc.set_b(b0)
    assert conv_g and conv_o and it_g == it_o
    st = ssg.stepforward_(prob, 100)
    orc.step(100)
    assert st.ma_unconverged == 0 and st.ma_iterations == orc.stats()["total_iters"] - it_o
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-10
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-10
    prob.close()
    orc.close()


def test_config2_fp64_512x32_rk3(require_gpu, ssg, oracle_mod, record_property):
    """Configuration 2 (the FP64 drop-in): 512^2 x 32, RK3, dt 5e-4, k0 = 10.
    20 steps against the oracle, with the oracle's time recorded."""
    n, nz, nsteps = 512, 32, 20
    dom, prob, orc = pair(ssg, oracle_mod, n, nz, "RK3", 5e-4, "quadratic")
    b0 = ssg.jfm_spectral_buoyancy(n, n, 10, seed=512)
    it_g, conv_g, _ = ssg.set_b_(prob, b0, dom)
    conv_o, it_o, _ = orc.set_b(b0)
    assert conv_g and conv_o and it_g == it_o
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-11
    st = ssg.stepforward_(prob, nsteps)
    t0 = time.perf_counter()
    orc.step(nsteps)
    t_orc = time.perf_counter() - t0
    record_property("oracle_steps_per_s", nsteps / t_orc)
    record_property("oracle_threads", oracle_mod.num_threads())
    print(f"config 2: oracle {nsteps / t_orc:.3f} steps/s on {oracle_mod.num_threads()} threads")
    assert st.ma_unconverged == 0
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-10
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-10
    assert rel(prob.fields.phi, orc.get(oracle_mod.FIELD_PHI)) < 1e-10
    t, step = orc.time()
    assert prob.clock.step == step == nsteps and abs(prob.clock.t - t) < 1e-15
    prob.close()
    orc.close()


def test_config3_fp64_1024x32(require_gpu, ssg, oracle_mod):
    """Configuration 3's grid in FP64: set_b and 5 AB2 steps against the
    oracle, and the converged potential's residual (the stop rule bounds the
    relative update at 1e-10; the residual of the projected equation, relative
    to ||b_s||, is measured at 1.1e-8 on this grid)."""
    n, nz = 1024, 32
    dom, prob, orc = pair(ssg, oracle_mod, n, nz, "AB2", 2.5e-4, "cubic")
    b0 = ssg.jfm_spectral_buoyancy(n, n, 16, seed=2024)
    it_g, conv_g, _ = ssg.set_b_(prob, b0, dom)
    conv_o, it_o, _ = orc.set_b(b0)
    assert conv_g and conv_o and it_g == it_o
    rint, rtop, rbot = ma_residual(prob.fields.phi, prob.fields.bs, 0.01)
    assert rint < 3e-8 and rtop < 1e-13 and rbot < 1e-13
    ssg.stepforward_(prob, 5)
    orc.step(5)
    assert rel(prob.fields.bs, orc.get(oracle_mod.FIELD_B_S)) < 1e-10
    assert rel(prob.fields.phis, orc.get(oracle_mod.FIELD_PHI_S)) < 1e-10
    prob.close()
    orc.close()


@pytest.mark.parametrize("seed,k0", [(2024, 16), (7, 16), (2024, 24)])
def test_config3_mixed_error_1000_steps(require_gpu, ssg, seed, k0):
    """Configuration 3: the mixed-precision path (FP32 Monge-Ampere
    transforms, FP64 solve and accumulation) stays within 1e-6 relative L2 of
    the FP64 GPU path after 10, 100 and 1000 AB2 steps at 1024^2 x 32."""
    n, nz = 1024, 32
    checkpoints = (10, 100, 1000)
    out = {}
    for prec in ("fp64", "mixed"):
        dom = ssg.make_domain(n, n, nz)
        prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.AB2_LowStorage, dt=2.5e-4, eps=0.01, filter_freq=10,
                                          filter_order=8, filter_strength=0.1, filter_cutoff=0.65, ma_tol=1e-10,
                                          precision=prec, enable_diagnostics=False)
        ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, k0, seed=seed), dom)
        done, res = 0, []
        for c in checkpoints:
            st = ssg.stepforward_(prob, c - done)
            assert st.ma_unconverged == 0
            done = c
            res.append(prob.fields.bs)
        if prec == "mixed":
            # FP32 transforms leave the converged residual near 1e-3 of ||b_s||
            # (measured 1.1e-3), against 1e-8 in FP64
            rint, _, _ = ma_residual(prob.fields.phi, res[-1], 0.01)
            assert rint < 1e-2
        out[prec] = res
        prob.close()
    errs = [rel(m, f) for m, f in zip(out["mixed"], out["fp64"])]
    print(f"mixed vs fp64 (seed {seed}, k0 {k0}): " + ", ".join(f"{e:.2e}" for e in errs))
    assert all(e < 1e-6 for e in errs), errs


def test_full_size_residual_after_steps(require_gpu, ssg):
    """After 20 AB2 steps at 1024^2 x 32 the potential each step solves for
    still satisfies the projected equation and both Neumann rows."""
    n, nz = 1024, 32
    dom = ssg.make_domain(n, n, nz)
    prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.AB2_LowStorage, dt=2.5e-4, filter_order=8,
                                      enable_diagnostics=False)
    ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 16, seed=2024), dom)
    ssg.stepforward_(prob, 20)
    rint, rtop, rbot = ma_residual(prob.fields.phi, prob.fields.bs, 0.01)
    assert rint < 3e-8 and rtop < 1e-13 and rbot < 1e-13
    prob.close()
