"""The register-resident vertical solve (ma_thomas_reg_kernel, compile-time
depths 8, 12, 16, 24 and 32) against the shared-memory staged one
(SSG_B200_THOMAS_STAGED=1, every depth): the same operations in the same
order, so fields, potentials and iteration counts are bit-identical.  The
update norm is summed over blocks of 64 modes instead of 32, so it agrees to
rounding only.

The transposed solve of the adjoint has the same two forms: the register
kernel solves A^T from the forward pivot table (no divisions), the staged one
factors A^T itself, so gradients agree to rounding."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make(ssg, n, nz, precision, scheme, staged, rhs="surface", **kw):
    old = os.environ.get("SSG_B200_THOMAS_STAGED")
    os.environ["SSG_B200_THOMAS_STAGED"] = "1" if staged else "0"
    try:
        dom = ssg.make_domain(n, n, nz)
        prob = ssg.SemiGeostrophicProblem(dom, scheme=scheme, dt=1e-3, filter_freq=4, filter_order=8,
                                          precision=precision, ma_rhs=rhs, enable_diagnostics=False, **kw)
    finally:
        if old is None:
            del os.environ["SSG_B200_THOMAS_STAGED"]
        else:
            os.environ["SSG_B200_THOMAS_STAGED"] = old
    return dom, prob


def run(ssg, n, nz, precision, scheme, staged, rhs="surface"):
    dom, prob = make(ssg, n, nz, precision, scheme, staged, rhs)
    it0 = ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 4, seed=91 + nz), dom)
    st = ssg.stepforward_(prob, 6)
    out = (prob.fields.bs, prob.fields.phi, it0[0], st.ma_iterations, it0[2])
    prob.close()
    return out


@pytest.mark.parametrize("nz", [8, 12, 16, 24, 32])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_register_solve_is_bit_identical(require_gpu, ssg, nz, precision):
    a = run(ssg, 64, nz, precision, ssg.AB2_LowStorage, staged=True)
    b = run(ssg, 64, nz, precision, ssg.AB2_LowStorage, staged=False)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert a[2:4] == b[2:4]
    assert abs(a[4] - b[4]) <= 1e-12 * abs(a[4])


def test_register_solve_rk3_volume_rhs(require_gpu, ssg):
    a = run(ssg, 128, 16, "fp64", ssg.RK3, staged=True, rhs="volume")
    b = run(ssg, 128, 16, "fp64", ssg.RK3, staged=False, rhs="volume")
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2:4] == b[2:4]


@pytest.mark.parametrize("nz,rhs,scheme", [(16, "surface", "RK3"), (12, "volume", "AB2"), (32, "surface", "AB2")])
def test_transposed_solve_forms_agree(require_gpu, ssg, nz, rhs, scheme):
    n = 64
    sch = ssg.RK3 if scheme == "RK3" else ssg.AB2_LowStorage
    b0 = ssg.jfm_spectral_buoyancy(n, n, 5, seed=41)
    target = ssg.jfm_spectral_buoyancy(n, n, 5, seed=42)
    grads = []
    for staged in (True, False):
        dom, prob = make(ssg, n, nz, "fp64", sch, staged, rhs, ma_tol=1e-13, ma_maxiter=200)
        L, g = ssg.adjoint.misfit_loss_and_gradient(prob, b0, target, 10, 4)
        grads.append((L, g))
        prob.close()
    (La, ga), (Lb, gb) = grads
    assert La == Lb
    assert np.abs(ga - gb).max() <= 1e-11 * np.abs(ga).max()
