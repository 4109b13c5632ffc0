"""The register-resident vertical solve (ma_thomas_reg_kernel, compile-time
depths 8, 12, 16, 24 and 32) against the shared-memory staged one
(SSG_B200_THOMAS_STAGED=1, every depth): the same operations in the same
order, so fields, potentials and iteration counts are bit-identical.  The
update norm is summed over blocks of 64 modes instead of 32, so it agrees to
rounding only."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(ssg, n, nz, precision, scheme, staged, rhs="surface"):
    old = os.environ.get("SSG_B200_THOMAS_STAGED")
    os.environ["SSG_B200_THOMAS_STAGED"] = "1" if staged else "0"
    try:
        dom = ssg.make_domain(n, n, nz)
        prob = ssg.SemiGeostrophicProblem(dom, scheme=scheme, dt=1e-3, filter_freq=4, filter_order=8,
                                          precision=precision, ma_rhs=rhs, enable_diagnostics=False)
    finally:
        if old is None:
            del os.environ["SSG_B200_THOMAS_STAGED"]
        else:
            os.environ["SSG_B200_THOMAS_STAGED"] = old
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
