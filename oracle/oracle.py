"""ctypes wrapper around liboracle_ssg.so, the CPU restatement of SSG.jl's
time-step path.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the CPU-baseline leg of bench.py, where it is the checker (or the timed CPU
baseline), never the thing measured on the GPU.

Arrays follow the reference's Julia layout: a 2-D field b[i, j] is a
Fortran-ordered (nx, ny) float64 array, a 3-D field Phi[i, j, k] a
Fortran-ordered (nx, ny, nz) array (x fastest in memory).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_ssg.so")

FIELD_B_S, FIELD_PHI_S, FIELD_PHI, FIELD_DBDT_OLD, FIELD_U_S, FIELD_V_S = range(6)


class OrConfig(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("scheme", ctypes.c_int32),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("eps", ctypes.c_double), ("dt", ctypes.c_double),
        ("filter_freq", ctypes.c_int32), ("filter_order", ctypes.c_int32),
        ("filter_strength", ctypes.c_double), ("filter_cutoff", ctypes.c_double),
        ("ma_tol", ctypes.c_double),
        ("ma_maxiter", ctypes.c_int32), ("ma_per_stage", ctypes.c_int32),
        ("ma_rhs_mode", ctypes.c_int32), ("ma_predictor", ctypes.c_int32),
        ("filter_type", ctypes.c_int32), ("ab2_literal_alias", ctypes.c_int32),
        ("ma_bc_guess", ctypes.c_int32), ("pad2", ctypes.c_int32),
    ]


class OrStats(ctypes.Structure):
    _fields_ = [
        ("last_iters", ctypes.c_int32), ("total_iters", ctypes.c_int32),
        ("max_iters", ctypes.c_int32), ("solves", ctypes.c_int32),
        ("unconverged", ctypes.c_int32), ("pad0", ctypes.c_int32),
        ("last_update", ctypes.c_double), ("max_update", ctypes.c_double),
    ]


_lib = None


def build():
    """Compile liboracle_ssg.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.or_create.restype = P
        L.or_create.argtypes = [ctypes.POINTER(OrConfig)]
        L.or_destroy.argtypes = [P]
        L.or_set_dz.argtypes = [P, dp]
        L.or_set_b.argtypes = [P, dp, ip, dp]
        L.or_solve_ma.argtypes = [P, ip, dp]
        L.or_step.argtypes = [P, ctypes.c_int, ctypes.c_double]
        L.or_get_stats.argtypes = [P, ctypes.POINTER(OrStats)]
        L.or_get_time.argtypes = [P, dp, ctypes.POINTER(ctypes.c_long)]
        L.or_set_time.argtypes = [P, ctypes.c_double, ctypes.c_long]
        L.or_get_field.argtypes = [P, ctypes.c_int, dp]
        L.or_set_field.argtypes = [P, ctypes.c_int, dp]
        L.or_rfft2.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        L.or_irfft2.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        L.or_jacobian.argtypes = [P, dp, dp, dp]
        L.or_tendency.argtypes = [P, dp, dp, dp]
        L.or_exponential_transfer.restype = ctypes.c_double
        L.or_exponential_transfer.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double]
        L.or_filter.argtypes = [P, dp]
        L.or_grid_tables.argtypes = [P, dp, dp, ctypes.POINTER(ctypes.c_uint8)]
        L.or_ssg_residual_literal.argtypes = [P, dp, dp, dp, ctypes.c_double, dp]
        L.or_mg_create.restype = P
        L.or_mg_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int]
        L.or_mg_destroy.argtypes = [P]
        L.or_mg_set_dz.argtypes = [P, dp]
        L.or_mg_level_nx.argtypes = [P, ctypes.c_int]
        L.or_mg_set.argtypes = [P, ctypes.c_int, ctypes.c_int, dp]
        L.or_mg_get.argtypes = [P, ctypes.c_int, ctypes.c_int, dp]
        L.or_mg_residual.argtypes = [P, ctypes.c_int, ctypes.c_double]
        L.or_mg_boundary.argtypes = [P, ctypes.c_int]
        L.or_mg_smooth.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.or_mg_restrict.argtypes = [P, ctypes.c_int]
        L.or_mg_prolongate.argtypes = [P, ctypes.c_int]
        L.or_mg_v_cycle.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.or_mg_norm.restype = ctypes.c_double
        L.or_mg_norm.argtypes = [P, ctypes.c_int, ctypes.c_int]
        L.or_mg_solve.restype = ctypes.c_int
        L.or_mg_solve.argtypes = [P, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  ctypes.POINTER(ctypes.c_int), dp]
        L.or_num_threads.restype = ctypes.c_int
        L.or_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f2(a, nx, ny):
    a = np.asarray(a, dtype=np.float64)
    assert a.shape == (nx, ny), a.shape
    return np.asfortranarray(a)


def rfft2(b):
    """rfft_2d!: (nx, ny) real -> (nx, ny//2+1) complex, unnormalised."""
    b = np.asfortranarray(np.asarray(b, dtype=np.float64))
    nx, ny = b.shape
    out = np.zeros((nx, ny // 2 + 1), dtype=np.complex128, order="F")
    lib().or_rfft2(nx, ny, _dp(b), _dp(out))
    return out


def irfft2(s, ny):
    """irfft_2d!: (nx, ny//2+1) complex -> (nx, ny) real, scaled 1/(nx ny)."""
    s = np.asfortranarray(np.asarray(s, dtype=np.complex128))
    nx = s.shape[0]
    out = np.zeros((nx, ny), dtype=np.float64, order="F")
    lib().or_irfft2(nx, ny, _dp(s), _dp(out))
    return out


def exponential_transfer(knorm, strength, order, cutoff):
    return lib().or_exponential_transfer(knorm, strength, order, cutoff)


class Oracle:
    """CPU restatement of one SemiGeostrophicProblem (single member)."""

    def __init__(self, nx, ny, nz, *, lx=2 * np.pi, ly=2 * np.pi, lz=1.0, eps=0.01,
                 dt=1e-3, scheme=0, filter_freq=10, filter_order=8,
                 filter_strength=0.1, filter_cutoff=0.65, ma_tol=1e-10,
                 ma_maxiter=50, ma_per_stage=1, ma_rhs_mode=0, ma_predictor=3, filter_type=0, dz=None,
                 ab2_literal_alias=0, ma_bc_guess=1):
        self.cfg = OrConfig(nx, ny, nz, scheme, lx, ly, lz, eps, dt, filter_freq,
                            filter_order, filter_strength, filter_cutoff, ma_tol,
                            ma_maxiter, ma_per_stage, ma_rhs_mode, ma_predictor, filter_type,
                            1 if ab2_literal_alias else 0, 1 if ma_bc_guess else 0, 0)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.h = lib().or_create(ctypes.byref(self.cfg))
        if not self.h:
            raise ValueError("oracle: unsupported configuration")
        if dz is not None:
            # Domain.dz of a stretched or custom grid (src/domain.jl:238-280)
            d = np.ascontiguousarray(dz, dtype=np.float64)
            if d.size != nz:
                raise ValueError("oracle: dz needs nz values")
            lib().or_set_dz(self.h, _dp(d))

    def close(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_b(self, b):
        b = _f2(b, self.nx, self.ny)
        it = ctypes.c_int(0)
        upd = ctypes.c_double(0)
        rc = lib().or_set_b(self.h, _dp(b), ctypes.byref(it), ctypes.byref(upd))
        return rc == 0, it.value, upd.value

    def solve_ma(self):
        it = ctypes.c_int(0)
        upd = ctypes.c_double(0)
        rc = lib().or_solve_ma(self.h, ctypes.byref(it), ctypes.byref(upd))
        return rc == 0, it.value, upd.value

    def step(self, n=1, dt=0.0):
        lib().or_step(self.h, int(n), float(dt))

    def stats(self):
        s = OrStats()
        lib().or_get_stats(self.h, ctypes.byref(s))
        return {f: getattr(s, f) for f, _ in OrStats._fields_ if f != "pad0"}

    def time(self):
        t = ctypes.c_double(0)
        st = ctypes.c_long(0)
        lib().or_get_time(self.h, ctypes.byref(t), ctypes.byref(st))
        return t.value, st.value

    def set_time(self, t, step):
        lib().or_set_time(self.h, float(t), int(step))

    def get(self, field):
        if field == FIELD_PHI:
            out = np.zeros((self.nx, self.ny, self.nz), order="F")
        else:
            out = np.zeros((self.nx, self.ny), order="F")
        rc = lib().or_get_field(self.h, field, _dp(out))
        if rc != 0:
            raise ValueError("oracle: bad field id")
        return out

    def set(self, field, arr):
        a = _f2(arr, self.nx, self.ny)
        if lib().or_set_field(self.h, field, _dp(a)) != 0:
            raise ValueError("oracle: bad field id")

    def jacobian(self, phi, b):
        phi = _f2(phi, self.nx, self.ny)
        b = _f2(b, self.nx, self.ny)
        out = np.zeros((self.nx, self.ny), order="F")
        lib().or_jacobian(self.h, _dp(phi), _dp(b), _dp(out))
        return out

    def tendency(self, phi, b):
        phi = _f2(phi, self.nx, self.ny)
        b = _f2(b, self.nx, self.ny)
        out = np.zeros((self.nx, self.ny), order="F")
        lib().or_tendency(self.h, _dp(phi), _dp(b), _dp(out))
        return out

    def filter(self, b):
        out = np.array(_f2(b, self.nx, self.ny), order="F", copy=True)
        lib().or_filter(self.h, _dp(out))
        return out

    def grid_tables(self):
        nyc = self.ny // 2 + 1
        kx = np.zeros(self.nx)
        ky = np.zeros(nyc)
        mask = np.zeros((self.nx, nyc), dtype=np.uint8, order="F")
        lib().or_grid_tables(self.h, _dp(kx), _dp(ky), mask.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        return kx, ky, mask.astype(bool)

    def ssg_residual_literal(self, Phi, rhs, bs_surface, eps):
        Phi = np.array(Phi, dtype=np.float64, order="F", copy=True)
        rhs = np.asfortranarray(np.asarray(rhs, dtype=np.float64))
        bs = _f2(bs_surface, self.nx, self.ny)
        r = np.zeros_like(Phi, order="F")
        lib().or_ssg_residual_literal(self.h, _dp(Phi), _dp(rhs), _dp(bs), float(eps), _dp(r))
        return Phi, r


def num_threads():
    return lib().or_num_threads()


def set_num_threads(n):
    lib().or_set_num_threads(int(n))


MG_PHI, MG_RHS, MG_RESIDUAL, MG_BS_SURFACE = range(4)
SMOOTHER_SPECTRAL, SMOOTHER_SOR, SMOOTHER_ENHANCED = range(3)


class OracleMG:
    """The reference's multigrid hierarchy (SSGMultigridSolver + SSGLevel),
    restated literally on the CPU."""

    def __init__(self, nx, ny, nz, *, lx=2 * np.pi, ly=2 * np.pi, lz=1.0, n_levels=3, dz=None):
        self.h = lib().or_mg_create(nx, ny, nz, lx, ly, lz, n_levels)
        if not self.h:
            raise ValueError("oracle: bad multigrid shape")
        if dz is not None:
            d = np.ascontiguousarray(dz, dtype=np.float64)
            if d.size != nz:
                raise ValueError("oracle: dz needs nz values")
            lib().or_mg_set_dz(self.h, _dp(d))
        self.nz, self.n_levels = nz, n_levels

    def close(self):
        if getattr(self, "h", None):
            lib().or_mg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def shape(self, level):
        n = lib().or_mg_level_nx(self.h, level)
        return n, n, self.nz

    def set(self, level, field, arr):
        nx, ny, nz = self.shape(level)
        shp = (nx, ny) if field == MG_BS_SURFACE else (nx, ny, nz)
        a = np.asfortranarray(np.asarray(arr, dtype=np.float64).reshape(shp, order="F"))
        lib().or_mg_set(self.h, level, field, _dp(a))

    def get(self, level, field):
        nx, ny, nz = self.shape(level)
        out = np.zeros((nx, ny) if field == MG_BS_SURFACE else (nx, ny, nz), order="F")
        lib().or_mg_get(self.h, level, field, _dp(out))
        return out

    def residual(self, level, eps):
        lib().or_mg_residual(self.h, level, eps)

    def boundary(self, level):
        lib().or_mg_boundary(self.h, level)

    def smooth(self, level, smoother, iters, omega, eps):
        lib().or_mg_smooth(self.h, level, smoother, iters, omega, eps)

    def restrict(self, coarse_level):
        lib().or_mg_restrict(self.h, coarse_level)

    def prolongate(self, coarse_level):
        lib().or_mg_prolongate(self.h, coarse_level)

    def v_cycle(self, smoother, omega, eps):
        lib().or_mg_v_cycle(self.h, smoother, omega, eps)

    def norm(self, level, field):
        return lib().or_mg_norm(self.h, level, field)

    def solve(self, eps, tol, maxiter, smoother, omega):
        it = ctypes.c_int(0)
        res = ctypes.c_double(0)
        conv = lib().or_mg_solve(self.h, eps, tol, maxiter, smoother, omega, ctypes.byref(it), ctypes.byref(res))
        return bool(conv), it.value, res.value
