"""ssg_tendency_noalloc against the time-step path.

The entry point serves callers that cannot allocate device memory: their
device memory belongs to a framework's pool or caching allocator, or they run
in loops where cudaMalloc's device synchronisation is not acceptable.  It
computes compute_tendency! on caller-owned device buffers, using a static
device array as its only working storage.

The check: for a field b and its streamfunction phi_s, one forward-Euler step
of the existing entry points (ssg_set_b, then ssg_step with dt = 1, phi_s
frozen, no filter) gives b + f; the no-alloc entry point must return the same
f.  Two calls in a row, on two different fields, both checked.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


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


def test_noalloc_tendency_matches_time_step(require_gpu, ssg):
    import torch

    L = ssg._lib.load()
    n = 128
    two_pi = 2 * np.pi
    # sizes beyond the static array are rejected before any device work
    assert L.ssg_tendency_noalloc(1024, 1024, two_pi, two_pi, 1, 1, 1, None) == ssg._lib.SSG_ERR_ARG
    assert b"512" in L.ssg_last_error(None)
    for seed in (11, 12):
        b0 = ssg.jfm_spectral_buoyancy(n, n, 6, seed=seed)
        phi, b, f_ref = tendency_through_step(ssg, n, b0)
        d_phi = torch.from_numpy(phi.ravel(order="F").copy()).cuda()
        d_b = torch.from_numpy(b.ravel(order="F").copy()).cuda()
        d_f = torch.full_like(d_b, float("nan"))
        torch.cuda.synchronize()
        rc = L.ssg_tendency_noalloc(n, n, two_pi, two_pi, d_phi.data_ptr(), d_b.data_ptr(), d_f.data_ptr(), None)
        assert rc == ssg._lib.SSG_OK
        torch.cuda.synchronize()
        f = d_f.cpu().numpy().reshape((n, n), order="F")
        assert np.isfinite(f).all()
        assert rel(f, f_ref) < 1e-12, (seed, rel(f, f_ref))
