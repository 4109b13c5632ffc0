"""The reference's own Monge-Ampere multigrid (src/poisson.jl:33-959) on the GPU.

``SSGMultigrid`` is SSGMultigridSolver's hierarchy of SSGLevels; its methods
are compute_ssg_residual!, apply_ssg_boundary_conditions!, the spectral and
red-black SOR smoothers, the injection transfers, ssg_v_cycle! and
norm_field.  ``solve_ssg_equation`` is the reference's driver.  They reproduce
SSG.jl as written: the spectral smoother diverges and the SOR smoother
ignores the right-hand side.  The time step solves the documented equations
with ``solve_monge_ampere_fields_`` instead.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, load

SMOOTHERS = {"spectral": _lib.SMOOTHER_SPECTRAL, "sor": _lib.SMOOTHER_SOR, "enhanced": _lib.SMOOTHER_ENHANCED,
             "adaptive": _lib.SMOOTHER_ADAPTIVE}
FIELDS = {"phi": _lib.MG_PHI, "b": _lib.MG_RHS, "r": _lib.MG_RESIDUAL, "bs_surface": _lib.MG_BS_SURFACE}


def _mg_check(rc, h, allow=()):
    if rc == _lib.SSG_OK or rc in allow:
        return rc
    msg = load().ssg_mg_last_error(h)
    raise _lib.SsgError(rc, msg.decode() if msg else "")


class SSGMultigrid:
    """SSGMultigridSolver's levels on one device.  A custom vertical grid
    carries to every level (create_coarse_domain keeps nz and passes z,
    src/coarse_domain.jl:55-65).  A stretched grid with more than one level
    raises, as the reference's coarse-domain constructor does: it passes no
    stretch_params for a stretched grid and make_vertical_grid rejects that."""

    def __init__(self, domain, n_levels=3, device=0):
        grid = getattr(domain, "z_grid", "uniform")
        if grid == "stretched" and n_levels > 1:
            raise ValueError("stretch_params required for 'stretched' grid (coarse levels of a stretched grid)")
        L = load()
        h = ctypes.c_void_p()
        rc = L.ssg_mg_create(domain.Nx, domain.Ny, domain.Nz, domain.Lx, domain.Ly, domain.Lz, n_levels, device,
                             ctypes.byref(h))
        _mg_check(rc, None)
        self.h = h
        self.n_levels = n_levels
        if grid != "uniform":
            dz = np.ascontiguousarray(domain.dz, dtype=np.float64)
            _mg_check(L.ssg_mg_set_vertical_grid(h, dz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), dz.size), h)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            load().ssg_mg_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, level):
        nx, ny, nz = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _mg_check(load().ssg_mg_level_shape(self.h, level, ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(nz)),
                  self.h)
        return nx.value, ny.value, nz.value

    def _shape_of(self, level, field):
        nx, ny, nz = self.shape(level)
        return (nx, ny) if field == "bs_surface" else (nx, ny, nz)

    def set(self, level, field, arr):
        a = np.asfortranarray(np.asarray(arr, dtype=np.float64))
        if a.shape != self._shape_of(level, field):
            raise ValueError(f"expected {self._shape_of(level, field)}, got {a.shape}")
        _mg_check(load().ssg_mg_set(self.h, level, FIELDS[field], a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                    a.size), self.h)

    def get(self, level, field):
        out = np.empty(self._shape_of(level, field), dtype=np.float64, order="F")
        _mg_check(load().ssg_mg_get(self.h, level, FIELDS[field],
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size), self.h)
        return out

    def residual(self, level, eps):
        _mg_check(load().ssg_mg_residual(self.h, level, eps), self.h)

    def boundary(self, level):
        _mg_check(load().ssg_mg_boundary(self.h, level), self.h)

    def smooth(self, level, smoother, iters, omega, eps):
        _mg_check(load().ssg_mg_smooth(self.h, level, SMOOTHERS[smoother], iters, omega, eps), self.h)

    def restrict(self, coarse_level):
        _mg_check(load().ssg_mg_restrict(self.h, coarse_level), self.h)

    def prolongate(self, coarse_level):
        _mg_check(load().ssg_mg_prolongate(self.h, coarse_level), self.h)

    def v_cycle(self, smoother, omega, eps):
        _mg_check(load().ssg_mg_v_cycle(self.h, SMOOTHERS[smoother], omega, eps), self.h)

    def norm(self, level, field):
        out = ctypes.c_double()
        _mg_check(load().ssg_mg_norm(self.h, level, FIELDS[field], ctypes.byref(out)), self.h)
        return out.value


def solve_ssg_equation(Phi_initial, b_rhs, eps, domain, *, tol=1e-8, maxiter=50, verbose=False, n_levels=3,
                       smoother="spectral", omega=0.8, device=0):
    """solve_ssg_equation (src/poisson.jl:869-959): returns (solution,
    diagnostics) like the reference (converged, iterations, final_residual,
    eps_parameter)."""
    mg = SSGMultigrid(domain, n_levels, device)
    mg.set(0, "phi", Phi_initial)
    mg.set(0, "b", b_rhs)
    it, res, conv = ctypes.c_int32(), ctypes.c_double(), ctypes.c_int32()
    rc = load().ssg_mg_solve(mg.h, eps, tol, maxiter, SMOOTHERS[smoother], omega, ctypes.byref(it),
                             ctypes.byref(res), ctypes.byref(conv))
    _mg_check(rc, mg.h, allow=(_lib.SSG_ERR_NOT_CONVERGED,))
    sol = mg.get(0, "phi")
    if verbose:
        print(f"[SSG] {it.value} V-cycles, residual {res.value:.3e}")
    mg.close()
    return sol, dict(converged=bool(conv.value), iterations=it.value, final_residual=res.value, eps_parameter=eps)
