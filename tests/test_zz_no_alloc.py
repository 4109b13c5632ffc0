"""ssg_tendency_noalloc, the tendency entry point that allocates nothing.

It serves callers that cannot allocate device memory: their device memory
belongs to a framework's pool or caching allocator, or they run in loops where
cudaMalloc's device synchronisation is not acceptable.  It computes
compute_tendency! on caller-owned device buffers, using a static device array
as its only working storage.

Checks, through the C ABI:
  * against the CPU oracle's compute_tendency! at the smallest grid (32), a
    middle one (128) and the largest the static array holds (512);
  * against the existing entry points: one forward-Euler step of ssg_step
    (dt = 1, phi_s frozen, no filter) from the same fields gives b + f;
  * calls in a row on alternating grids (each call writes its own tables);
  * grids beyond the array and non-square grids are rejected.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TWO_PI = 2 * np.pi


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def noalloc(L, ssg, phi, b):
    import torch

    n = phi.shape[0]
    d_phi = torch.from_numpy(phi.ravel(order="F").copy()).cuda()
    d_b = torch.from_numpy(b.ravel(order="F").copy()).cuda()
    d_f = torch.full_like(d_b, float("nan"))
    torch.cuda.synchronize()
    rc = L.ssg_tendency_noalloc(n, n, TWO_PI, TWO_PI, d_phi.data_ptr(), d_b.data_ptr(), d_f.data_ptr(), None)
    assert rc == ssg._lib.SSG_OK, L.ssg_last_error(None)
    torch.cuda.synchronize()
    f = d_f.cpu().numpy().reshape((n, n), order="F")
    assert np.isfinite(f).all()
    return f


def tendency_through_step(ssg, n, b0):
    dom = ssg.make_domain(n, n, 8)
    prob = ssg.SemiGeostrophicProblem(dom, scheme=ssg.AB2_LowStorage, dt=1.0, ma_per_stage=False, filter_freq=0,
                                      enable_diagnostics=False)
    ssg.set_b_(prob, b0, dom)
    b = prob.fields.bs
    phi = prob.fields.phis
    ssg.stepforward_(prob, 1)
    f = prob.fields.bs - b
    prob.close()
    return phi, b, f


def test_noalloc_tendency_matches_oracle(require_gpu, ssg, oracle_mod):
    L = ssg._lib.load()
    # sizes beyond the static array, and non-square grids, are rejected before any device work
    assert L.ssg_tendency_noalloc(1024, 1024, TWO_PI, TWO_PI, 1, 1, 1, None) == ssg._lib.SSG_ERR_ARG
    assert b"512" in L.ssg_last_error(None)
    assert L.ssg_tendency_noalloc(128, 64, TWO_PI, TWO_PI, 1, 1, 1, None) == ssg._lib.SSG_ERR_ARG
    for n, k0 in ((32, 4), (128, 6), (512, 10)):
        orc = oracle_mod.Oracle(n, n, 4)
        for seed in (3, 4):   # two calls in a row on the same grid
            phi = 0.2 * ssg.jfm_spectral_buoyancy(n, n, k0, seed=100 * seed + n)
            b = ssg.jfm_spectral_buoyancy(n, n, k0, seed=100 * seed + n + 1)
            f = noalloc(L, ssg, phi, b)
            assert rel(f, orc.tendency(phi, b)) < 1e-12, (n, seed)
        orc.close()


def test_noalloc_tendency_matches_time_step(require_gpu, ssg):
    L = ssg._lib.load()
    # alternating grids: every call carries its own tables into the array
    for n, seed in ((128, 11), (64, 12), (128, 13), (64, 14)):
        b0 = ssg.jfm_spectral_buoyancy(n, n, 6, seed=seed)
        phi, b, f_ref = tendency_through_step(ssg, n, b0)
        f = noalloc(L, ssg, phi, b)
        assert rel(f, f_ref) < 1e-12, (n, seed, rel(f, f_ref))
