"""ctypes binding of libssg_b200.so (declared in include/ssg_b200.h).

The library is built in-tree (``make -C ssg.jl_b200``) and loaded from this
directory.  There is no fallback: if the library or a CUDA device is missing,
loading or context creation raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libssg_b200.so")

ABI_VERSION = 1

SSG_OK = 0
SSG_ERR_ARG = -1
SSG_ERR_CUDA = -2
SSG_ERR_NOT_CONVERGED = -3
SSG_ERR_NONFINITE = -4
SSG_ERR_OOM = -5
SSG_ERR_UNSUPPORTED = -6

STATUS_NAMES = {
    SSG_OK: "SSG_OK", SSG_ERR_ARG: "SSG_ERR_ARG", SSG_ERR_CUDA: "SSG_ERR_CUDA",
    SSG_ERR_NOT_CONVERGED: "SSG_ERR_NOT_CONVERGED", SSG_ERR_NONFINITE: "SSG_ERR_NONFINITE",
    SSG_ERR_OOM: "SSG_ERR_OOM", SSG_ERR_UNSUPPORTED: "SSG_ERR_UNSUPPORTED",
}

SCHEME_AB2, SCHEME_RK3 = 0, 1
MA_RHS_SURFACE, MA_RHS_VOLUME = 0, 1
FIELD_B_S, FIELD_PHI_S, FIELD_PHI, FIELD_DBDT_OLD, FIELD_U_S, FIELD_V_S = range(6)

# every symbol include/ssg_b200.h declares
EXPORTED_SYMBOLS = (
    "ssg_abi_version", "ssg_config_init", "ssg_ctx_create", "ssg_ctx_destroy",
    "ssg_set_b", "ssg_solve_ma", "ssg_step", "ssg_get_field", "ssg_set_field",
    "ssg_get_time", "ssg_set_time", "ssg_last_timing", "ssg_profile_kernels", "ssg_kernel_times",
    "ssg_tendency_noalloc", "ssg_apply_filter", "ssg_set_filter_table", "ssg_get_diagnostics",
    "ssg_checkpoint_size", "ssg_checkpoint", "ssg_restore", "ssg_mg_create", "ssg_mg_destroy",
    "ssg_mg_level_shape", "ssg_mg_set", "ssg_mg_get", "ssg_mg_residual", "ssg_mg_boundary", "ssg_mg_smooth",
    "ssg_mg_restrict", "ssg_mg_prolongate", "ssg_mg_v_cycle", "ssg_mg_norm", "ssg_mg_solve", "ssg_mg_last_error",
    "ssg_set_vertical_grid", "ssg_mg_set_vertical_grid", "ssg_adjoint_record", "ssg_adjoint", "ssg_ensemble_create", "ssg_ensemble_step", "ssg_ensemble_destroy",
    "ssg_ensemble_last_error", "ssg_members_gather", "ssg_members_scatter", "ssg_autotune", "ssg_set_tiles", "ssg_get_tiles", "ssg_set_variants",
    "ssg_get_variants", "ssg_last_error",
)
MG_PHI, MG_RHS, MG_RESIDUAL, MG_BS_SURFACE = range(4)
SMOOTHER_SPECTRAL, SMOOTHER_SOR, SMOOTHER_ENHANCED, SMOOTHER_ADAPTIVE = range(4)
FILTER_EXPONENTIAL, FILTER_HYPERVISCOSITY, FILTER_CUTOFF, FILTER_CESARO, FILTER_CUSTOM = range(5)
SSG_YPASS_PLAIN, SSG_YPASS_TMA, SSG_YPASS_WARP2, SSG_YPASS_WARP4, SSG_YPASS_WARP8 = 0, 1, 2, 4, 8
KERNEL_CLASSES = ("ma_xinv3", "ma_y", "ma_xfwd", "ma_thomas", "surf_xinv3", "surf_y", "surf_xfwd_stage", "field_io",
                  "adj_ma_xinv", "adj_ma_y", "adj_ma_xfwd", "adj_ma_thomas", "adj_surf")


class SsgConfig(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("eps", ctypes.c_double), ("dt", ctypes.c_double),
        ("scheme", ctypes.c_int32), ("filter_freq", ctypes.c_int32),
        ("filter_order", ctypes.c_int32), ("ma_maxiter", ctypes.c_int32),
        ("filter_strength", ctypes.c_double), ("filter_cutoff", ctypes.c_double),
        ("ma_tol", ctypes.c_double),
        ("ma_per_stage", ctypes.c_int32), ("ma_rhs_mode", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("ma_predictor", ctypes.c_int32), ("filter_type", ctypes.c_int32),
        ("ab2_literal_alias", ctypes.c_int32), ("ma_bc_guess", ctypes.c_int32),
        ("nmembers", ctypes.c_int32),
    ]


class SsgMaStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("converged", ctypes.c_int32), ("update", ctypes.c_double)]


class SsgStepStats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int32), ("ma_solves", ctypes.c_int32),
        ("ma_iterations", ctypes.c_int32), ("ma_iterations_max", ctypes.c_int32),
        ("ma_unconverged", ctypes.c_int32), ("pad0", ctypes.c_int32),
        ("ma_update_max", ctypes.c_double), ("t", ctypes.c_double), ("step", ctypes.c_int64),
    ]


class SsgDiagnostics(ctypes.Structure):
    _fields_ = [
        ("t", ctypes.c_double), ("step", ctypes.c_int64), ("kinetic_energy", ctypes.c_double),
        ("buoyancy_variance", ctypes.c_double), ("total_buoyancy", ctypes.c_double),
        ("ma_last_iterations", ctypes.c_int32), ("pad0", ctypes.c_int32),
    ]


class SsgAdjointStats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int32), ("checkpoints", ctypes.c_int32),
        ("forward_solves", ctypes.c_int32), ("forward_iterations", ctypes.c_int32),
        ("adjoint_solves", ctypes.c_int32), ("adjoint_iterations", ctypes.c_int32),
        ("adjoint_iterations_max", ctypes.c_int32), ("adjoint_unconverged", ctypes.c_int32),
        ("adjoint_update_max", ctypes.c_double), ("ms", ctypes.c_double), ("device_bytes", ctypes.c_int64),
    ]


class SsgError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def load():
    """Load libssg_b200.so and declare its signatures (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"libssg_b200.so not built (expected at {LIB_PATH}); run `make -C ssg.jl_b200`")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    L.ssg_abi_version.restype = ctypes.c_int
    L.ssg_config_init.argtypes = [ctypes.POINTER(SsgConfig)]
    L.ssg_config_init.restype = None
    L.ssg_ctx_create.argtypes = [ctypes.POINTER(SsgConfig), ctypes.c_int, ctypes.POINTER(vp)]
    L.ssg_ctx_destroy.argtypes = [vp]
    L.ssg_set_b.argtypes = [vp, dp, ctypes.c_int64, ctypes.POINTER(SsgMaStats)]
    L.ssg_solve_ma.argtypes = [vp, ctypes.POINTER(SsgMaStats)]
    L.ssg_step.argtypes = [vp, ctypes.c_int32, ctypes.c_double, ctypes.POINTER(SsgStepStats)]
    L.ssg_get_field.argtypes = [vp, ctypes.c_int32, dp, ctypes.c_int64]
    L.ssg_set_field.argtypes = [vp, ctypes.c_int32, dp, ctypes.c_int64]
    L.ssg_get_time.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int64)]
    L.ssg_set_time.argtypes = [vp, ctypes.c_double, ctypes.c_int64]
    L.ssg_last_timing.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int64)]
    L.ssg_profile_kernels.argtypes = [vp, ctypes.c_int]
    L.ssg_kernel_times.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int32]
    L.ssg_tendency_noalloc.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.ssg_apply_filter.argtypes = [vp]
    L.ssg_set_filter_table.argtypes = [vp, dp, ctypes.c_int64]
    L.ssg_get_diagnostics.argtypes = [vp, ctypes.POINTER(SsgDiagnostics)]
    L.ssg_checkpoint_size.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.ssg_checkpoint.argtypes = [vp, ctypes.c_void_p, ctypes.c_int64]
    L.ssg_restore.argtypes = [vp, ctypes.c_void_p, ctypes.c_int64]
    i32, dbl, pi32 = ctypes.c_int32, ctypes.c_double, ctypes.POINTER(ctypes.c_int32)
    L.ssg_mg_create.argtypes = [i32, i32, i32, dbl, dbl, dbl, i32, ctypes.c_int, ctypes.POINTER(vp)]
    L.ssg_mg_destroy.argtypes = [vp]
    L.ssg_mg_set_vertical_grid.argtypes = [vp, dp, i32]
    L.ssg_mg_level_shape.argtypes = [vp, i32, pi32, pi32, pi32]
    L.ssg_mg_set.argtypes = [vp, i32, i32, dp, ctypes.c_int64]
    L.ssg_mg_get.argtypes = [vp, i32, i32, dp, ctypes.c_int64]
    L.ssg_mg_residual.argtypes = [vp, i32, dbl]
    L.ssg_mg_boundary.argtypes = [vp, i32]
    L.ssg_mg_smooth.argtypes = [vp, i32, i32, i32, dbl, dbl]
    L.ssg_mg_restrict.argtypes = [vp, i32]
    L.ssg_mg_prolongate.argtypes = [vp, i32]
    L.ssg_mg_v_cycle.argtypes = [vp, i32, dbl, dbl]
    L.ssg_mg_norm.argtypes = [vp, i32, i32, dp]
    L.ssg_mg_solve.argtypes = [vp, dbl, dbl, i32, i32, dbl, pi32, dp, pi32]
    L.ssg_mg_last_error.argtypes = [vp]
    L.ssg_mg_last_error.restype = ctypes.c_char_p
    L.ssg_adjoint_record.argtypes = [vp, dp, ctypes.c_int64, i32, i32, ctypes.POINTER(SsgAdjointStats)]
    L.ssg_adjoint.argtypes = [vp, dp, dp, ctypes.c_int64, ctypes.POINTER(SsgAdjointStats)]
    L.ssg_autotune.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    L.ssg_set_tiles.argtypes = [vp, ctypes.c_int32, ctypes.c_int32]
    L.ssg_get_tiles.argtypes = [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    L.ssg_set_variants.argtypes = [vp, ctypes.c_int32, ctypes.c_int32]
    L.ssg_get_variants.argtypes = [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    L.ssg_set_vertical_grid.argtypes = [vp, dp, i32]
    L.ssg_ensemble_create.argtypes = [ctypes.POINTER(vp), i32, i32, ctypes.POINTER(vp)]
    L.ssg_ensemble_step.argtypes = [vp, i32, ctypes.POINTER(SsgStepStats)]
    L.ssg_members_gather.argtypes = [vp, ctypes.POINTER(vp), i32]
    L.ssg_members_scatter.argtypes = [vp, ctypes.POINTER(vp), i32]
    L.ssg_ensemble_destroy.argtypes = [vp]
    L.ssg_ensemble_last_error.argtypes = [vp]
    L.ssg_ensemble_last_error.restype = ctypes.c_char_p
    L.ssg_last_error.argtypes = [vp]
    L.ssg_last_error.restype = ctypes.c_char_p
    if L.ssg_abi_version() != ABI_VERSION:
        raise OSError("libssg_b200.so ABI version mismatch")
    _lib = L
    return L


def default_config():
    c = SsgConfig()
    load().ssg_config_init(ctypes.byref(c))
    return c


def check(rc, ctx=None, allow=()):
    if rc == SSG_OK or rc in allow:
        return rc
    msg = load().ssg_last_error(ctx)
    raise SsgError(rc, msg.decode() if msg else "")
