"""Host-side mirror of SSG.jl's public API for the time-step path.

Names follow SSG.jl (src/SSG.jl:41-80); Julia's mutating ``!`` suffix becomes a
trailing underscore (``set_b!`` -> ``set_b_``, ``timestep!`` -> ``timestep_``),
as in PyTorch's in-place convention.  Arrays use the reference's indexing:
a surface field is a Fortran-ordered ``(nx, ny)`` float64 array ``b[i, j]``
and the 3-D potential a Fortran-ordered ``(nx, ny, nz)`` array.

Everything below the API runs on one GPU through libssg_b200.so; the fields
live in device memory and are copied to the host only when read.  There is no
CPU fallback.  The MPI communicator of the reference collapses to one device:
``comm`` is accepted and ignored.
"""
import ctypes
import math

import numpy as np

from . import _lib
from ._lib import SsgConfig, SsgError, SsgMaStats, SsgStepStats, check, load

# TimeScheme (src/timestep.jl:10-14)
AB2_LowStorage = "AB2_LowStorage"
RK3 = "RK3"
RK3_LowStorage = "RK3_LowStorage"
_SCHEMES = {AB2_LowStorage: _lib.SCHEME_AB2, RK3: _lib.SCHEME_RK3}


def _param(params, *names, default):
    for n in names:
        if n in params:
            return params[n]
    return default


def _unit_nodes(n, lo=0.0):
    """range(lo, 1, length=n) for lo in {0, -1}: one correctly rounded
    division per node, as Julia's range computes them."""
    i = np.arange(n, dtype=np.float64)
    return i / (n - 1) if lo == 0.0 else (2.0 * i - (n - 1)) / (n - 1)


def _spacing(z):
    """Domain.dz from the node vector: dz[1] = z[2] - z[1], centred halves
    inside, dz[Nz] = z[Nz] - z[Nz-1] (src/domain.jl:269-274, 640-645)."""
    z = np.asarray(z, dtype=np.float64)
    dz = np.empty_like(z)
    dz[1:-1] = 0.5 * (z[2:] - z[:-2])
    dz[0] = z[1] - z[0]
    dz[-1] = z[-1] - z[-2]
    return dz


def create_stretched_grid(Nz, Lz, stretch_params):
    """create_stretched_grid (src/domain.jl:597-618) with the tanh, exponential,
    sinh and power-law maps of src/domain.jl:628-729.  ``stretch_params`` is a
    dict: ``type`` ("tanh" default), ``beta``/``β`` (2.0), ``alpha``/``α``
    (1.5), ``surface_concentration`` (True).  Returns (z, dz).  The formulas
    are the reference's as written: the surface-concentrated tanh grid runs
    from z = Lz down to 0 (negative spacings) and the surface-concentrated
    exponential grid does not start at 0."""
    kind = str(_param(stretch_params, "type", default="tanh")).lstrip(":")
    Lz = float(Lz)
    if kind in ("tanh", "exponential"):
        beta = float(_param(stretch_params, "beta", "β", default=2.0))
        surface = bool(_param(stretch_params, "surface_concentration", default=True))
        xi = _unit_nodes(Nz)
        if kind == "tanh":
            if surface:
                z = Lz * (1 - 0.5 * (1 + np.tanh(beta * (2 * xi - 1)) / math.tanh(beta)))
            else:
                z = Lz * 0.5 * (1 + np.tanh(beta * (2 * xi - 1)) / math.tanh(beta))
        elif surface:
            z = Lz * (1 - np.exp(-beta * xi) / (1 - math.exp(-beta)))
        else:
            z = Lz * (np.exp(beta * xi) - 1) / (math.exp(beta) - 1)
    elif kind == "sinh":
        beta = float(_param(stretch_params, "beta", "β", default=2.0))
        z = Lz * (0.5 + np.sinh(beta * _unit_nodes(Nz, -1.0)) / (2 * math.sinh(beta)))
    elif kind == "power":
        alpha = float(_param(stretch_params, "alpha", "α", default=1.5))
        z = Lz * _unit_nodes(Nz) ** alpha
    else:
        raise ValueError(f"Unknown stretch type: {kind}")
    return z, _spacing(z)


def make_vertical_grid(Nz, Lz, z_grid="uniform", z_boundary="dirichlet", stretch_params=None):
    """make_vertical_grid (src/domain.jl:238-280) -> (z, dz), both of length Nz.
    ``z_grid`` is "uniform", "stretched" (``stretch_params`` as for
    create_stretched_grid) or "custom" (``stretch_params={"z_coords": z}``)."""
    Nz, Lz = int(Nz), float(Lz)
    z_grid = str(z_grid).lstrip(":")
    if z_grid == "uniform":
        if z_boundary == "periodic":
            h = Lz / Nz
            return h * np.arange(Nz), np.full(Nz, h)
        return np.linspace(0.0, Lz, Nz), np.full(Nz, Lz / (Nz - 1))
    if z_grid == "stretched":
        if stretch_params is None:
            raise ValueError("stretch_params required for 'stretched' grid, e.g. {'type': 'tanh', 'beta': 2.0}")
        return create_stretched_grid(Nz, Lz, stretch_params)
    if z_grid == "custom":
        if stretch_params is None or "z_coords" not in stretch_params:
            raise ValueError("for a 'custom' grid, provide stretch_params={'z_coords': z}")
        z = np.array(stretch_params["z_coords"], dtype=np.float64).ravel()
        if z.size != Nz:
            raise ValueError(f"Custom z_coords length ({z.size}) must match Nz ({Nz})")
        return z, _spacing(z)
    raise ValueError(f"Unknown z_grid type: {z_grid}. Use 'uniform', 'stretched', or 'custom'")


class Domain:
    """Grid, wavenumbers and mask (src/domain.jl:33-186).  Host tables only:
    the device copies live in each problem's context.  Stretched and custom
    vertical grids enter the Monge-Ampere operator through ``dz``."""

    def __init__(self, Nx, Ny, Nz, *, Lx=2 * math.pi, Ly=2 * math.pi, Lz=1.0, z_boundary="dirichlet",
                 z_grid="uniform", stretch_params=None, comm=None):
        if z_boundary == "periodic":
            raise NotImplementedError("periodic z is not part of the Monge-Ampere problem")
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self.z_boundary, self.z_grid = z_boundary, str(z_grid).lstrip(":")
        self.stretch_params = dict(stretch_params) if stretch_params is not None else None
        dx, dy = self.Lx / self.Nx, self.Ly / self.Ny
        self.x = dx * np.arange(self.Nx)
        self.y = dy * np.arange(self.Ny)
        self.z, self.dz = make_vertical_grid(self.Nz, self.Lz, self.z_grid, z_boundary, stretch_params)
        from .ic import twothirds_mask, wavenumbers
        self.kx, self.ky = wavenumbers(self.Nx, self.Ny, self.Lx, self.Ly)
        KX, KY = np.meshgrid(self.kx, self.ky, indexing="ij")
        self.Krsq = KX ** 2 + KY ** 2
        with np.errstate(divide="ignore"):
            self.invKrsq = np.where(self.Krsq > 0, 1.0 / np.where(self.Krsq > 0, self.Krsq, 1.0), 0.0)
        self.mask = twothirds_mask(self.Nx, self.Ny // 2 + 1)
        self.aliased_fraction = 1.0 / 3.0

    def __repr__(self):
        return f"Domain({self.Nx}x{self.Ny}x{self.Nz}, L=({self.Lx:g}, {self.Ly:g}, {self.Lz:g}))"


def make_domain(Nx, Ny, Nz, *, Lx=2 * math.pi, Ly=2 * math.pi, Lz=1.0, z_boundary="dirichlet", z_grid="uniform",
                stretch_params=None, comm=None):
    """make_domain (src/domain.jl:217-230)."""
    return Domain(Nx, Ny, Nz, Lx=Lx, Ly=Ly, Lz=Lz, z_boundary=z_boundary, z_grid=z_grid,
                  stretch_params=stretch_params, comm=comm)


class TimeParams:
    """TimeParams (src/timestep.jl:19-40)."""

    def __init__(self, dt, *, scheme=AB2_LowStorage, filter_freq=10, filter_strength=0.1, cfl_safety=0.5,
                 max_dt=0.1, min_dt=1e-6, adaptive_dt=False):
        if scheme not in _SCHEMES:
            raise ValueError(f"Time integration scheme {scheme} not implemented yet")
        if adaptive_dt:
            raise NotImplementedError("adaptive_dt is not implemented on the GPU path")
        self.dt = float(dt)
        self.scheme = scheme
        self.filter_freq = int(filter_freq)
        self.filter_strength = float(filter_strength)
        self.cfl_safety, self.max_dt, self.min_dt = float(cfl_safety), float(max_dt), float(min_dt)
        self.adaptive_dt = False


class _Context:
    """Owns one ssg_ctx (device buffers + stream)."""

    def __init__(self, cfg, device):
        L = load()
        h = ctypes.c_void_p()
        rc = L.ssg_ctx_create(ctypes.byref(cfg), int(device), ctypes.byref(h))
        check(rc, None)
        self.h = h
        self.cfg = cfg
        self.device = int(device)
        self.n2 = cfg.nx * cfg.ny
        self.members = max(1, cfg.nmembers)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            load().ssg_ctx_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get(self, field, shape):
        out = np.empty(shape, dtype=np.float64, order="F")
        rc = load().ssg_get_field(self.h, field, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size)
        check(rc, self.h)
        return out

    def set(self, field, arr, shape):
        a = np.asfortranarray(np.asarray(arr, dtype=np.float64))
        if a.shape != shape:
            raise ValueError(f"expected shape {shape}, got {a.shape}")
        rc = load().ssg_set_field(self.h, field, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size)
        check(rc, self.h)

    def time(self):
        t = ctypes.c_double()
        s = ctypes.c_int64()
        check(load().ssg_get_time(self.h, ctypes.byref(t), ctypes.byref(s)), self.h)
        return t.value, s.value

    def set_time(self, t, step):
        check(load().ssg_set_time(self.h, float(t), int(step)), self.h)

    def step(self, n, dt):
        st = SsgStepStats()
        rc = load().ssg_step(self.h, int(n), float(dt), ctypes.byref(st))
        check(rc, self.h)
        return st

    def autotune(self, reps=3):
        x, y = ctypes.c_int32(), ctypes.c_int32()
        check(load().ssg_autotune(self.h, int(reps), ctypes.byref(x), ctypes.byref(y)), self.h)
        return x.value, y.value

    def set_tiles(self, x_threads, y_threads):
        check(load().ssg_set_tiles(self.h, int(x_threads), int(y_threads)), self.h)

    def tiles(self):
        x, y = ctypes.c_int32(), ctypes.c_int32()
        check(load().ssg_get_tiles(self.h, ctypes.byref(x), ctypes.byref(y)), self.h)
        return x.value, y.value

    def set_variants(self, y_pass, thomas_staged):
        check(load().ssg_set_variants(self.h, int(y_pass), int(thomas_staged)), self.h)

    def variants(self):
        y, t = ctypes.c_int32(), ctypes.c_int32()
        check(load().ssg_get_variants(self.h, ctypes.byref(y), ctypes.byref(t)), self.h)
        return y.value, t.value

    def solve_ma(self):
        st = SsgMaStats()
        rc = load().ssg_solve_ma(self.h, ctypes.byref(st))
        check(rc, self.h, allow=(_lib.SSG_ERR_NOT_CONVERGED,))
        return st

    def set_b(self, b):
        a = np.asfortranarray(np.asarray(b, dtype=np.float64))
        shape = (self.cfg.nx, self.cfg.ny) + ((self.members,) if self.members > 1 else ())
        if a.shape != shape:
            raise ValueError(f"expected shape {shape}, got {a.shape}")
        st = SsgMaStats()
        rc = load().ssg_set_b(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size, ctypes.byref(st))
        check(rc, self.h, allow=(_lib.SSG_ERR_NOT_CONVERGED,))
        return st

    def checkpoint(self):
        """The exact device state (ssg_checkpoint) as a byte array."""
        n = ctypes.c_int64()
        check(load().ssg_checkpoint_size(self.h, ctypes.byref(n)), self.h)
        blob = np.empty(n.value, dtype=np.uint8)
        check(load().ssg_checkpoint(self.h, blob.ctypes.data_as(ctypes.c_void_p), n.value), self.h)
        return blob

    def restore(self, blob):
        blob = np.ascontiguousarray(blob, dtype=np.uint8)
        check(load().ssg_restore(self.h, blob.ctypes.data_as(ctypes.c_void_p), blob.size), self.h)

    def last_timing(self):
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        check(load().ssg_last_timing(self.h, ctypes.byref(ms), ctypes.byref(n)), self.h)
        return ms.value, n.value


class Fields:
    """Device-resident Fields (src/fields.jl:28-60).  Reading an attribute
    copies the field to the host; assigning ``bs`` or ``db_dt_old`` copies
    it to the device (projected onto the 2/3-dealiased modes, which is the
    only part of the state the solver carries)."""

    def __init__(self, ctx, domain):
        self._ctx = ctx
        # ensemble members (nmembers > 1) along a last axis
        mem = (ctx.members,) if ctx.members > 1 else ()
        self._shape2 = (domain.Nx, domain.Ny) + mem
        self._shape3 = (domain.Nx, domain.Ny, domain.Nz) + mem

    @property
    def bs(self):
        return self._ctx.get(_lib.FIELD_B_S, self._shape2)

    @bs.setter
    def bs(self, value):
        self._ctx.set(_lib.FIELD_B_S, value, self._shape2)

    @property
    def phis(self):
        return self._ctx.get(_lib.FIELD_PHI_S, self._shape2)

    @property
    def phi(self):
        return self._ctx.get(_lib.FIELD_PHI, self._shape3)

    @property
    def u(self):
        """Surface u = -d(phi_s)/dy (compute_surface_geostrophic_velocities!)."""
        return self._ctx.get(_lib.FIELD_U_S, self._shape2)

    @property
    def v(self):
        """Surface v = d(phi_s)/dx."""
        return self._ctx.get(_lib.FIELD_V_S, self._shape2)

    # the reference's Unicode names (NFKC-normalised: bₛ == bs, φₛ == φs)
    @property
    def φs(self):
        return self.phis

    @property
    def φ(self):
        return self.phi


class TimeState:
    """TimeState (src/timestep.jl:45-86): the clock lives in the context."""

    def __init__(self, ctx, fields):
        self._ctx = ctx
        self._fields = fields

    @property
    def t(self):
        return self._ctx.time()[0]

    @t.setter
    def t(self, value):
        self._ctx.set_time(value, self.step)

    @property
    def step(self):
        return self._ctx.time()[1]

    @step.setter
    def step(self, value):
        self._ctx.set_time(self.t, value)

    @property
    def db_dt_old(self):
        return self._ctx.get(_lib.FIELD_DBDT_OLD, self._fields._shape2)

    @db_dt_old.setter
    def db_dt_old(self, value):
        self._ctx.set(_lib.FIELD_DBDT_OLD, value, self._fields._shape2)


class DiagnosticTimeSeries:
    """DiagnosticTimeSeries (src/timestep.jl:290-301), filled on the host."""

    def __init__(self):
        self.times, self.kinetic_energy, self.enstrophy = [], [], []
        self.total_buoyancy, self.max_divergence, self.max_cfl = [], [], []


def diagnostics(prob_or_fields):
    """Surface integrals computed on the device (ssg_get_diagnostics):
    kinetic_energy = 1/2 integral(u_s^2 + v_s^2), buoyancy_variance =
    integral(b_s^2), total_buoyancy = integral(b_s), over the Lx x Ly surface."""
    ctx = prob_or_fields._ctx
    d = _lib.SsgDiagnostics()
    check(load().ssg_get_diagnostics(ctx.h, ctypes.byref(d)), ctx.h)
    return {f: getattr(d, f) for f, _ in _lib.SsgDiagnostics._fields_ if f != "pad0"}


def update_diagnostics_(diag, fields, domain=None, state=None):
    """update_diagnostics! (src/timestep.jl:304-329) with true energies (the
    reference passes physical arrays to parsevalsum2, which scales them):
    the integrals come from a device reduction over the spectra."""
    d = diagnostics(fields)
    diag.times.append(d["t"])
    diag.kinetic_energy.append(d["kinetic_energy"])
    diag.enstrophy.append(0.0)
    diag.total_buoyancy.append(d["total_buoyancy"])
    diag.max_divergence.append(0.0)
    diag.max_cfl.append(0.0)
    return diag


class SemiGeostrophicProblem:
    """SemiGeostrophicProblem (src/timestep.jl:348-399) on one GPU.

    Keywords beyond the reference's: ``eps`` (Monge-Ampere epsilon), ``ma_tol``,
    ``ma_maxiter``, ``ma_per_stage`` (re-solve the streamfunction before every
    tendency; False keeps phi_s frozen after set_b_ as the reference's step
    does), ``ma_rhs`` ('surface' or 'volume'), ``ma_predictor`` (initial
    guess of each solve: 'previous' solution, 'extrapolate' linearly from
    the last two, 'quadratic' from the last three, 'cubic' from the last
    four; 'auto', the default, is cubic in FP64 and quadratic in mixed
    precision), ``precision`` ('fp64', or 'mixed': Monge-Ampere transforms
    in FP32, solve and accumulation in FP64), ``filter_order`` and
    ``filter_cutoff`` (the reference hard-codes 4 and 0.65),
    ``ab2_literal_alias`` (AB2 with the tendency the reference's
    timestep_ab2_ls! computes as written, -P[2 d/dy(b d(phi)/dx)], because it
    hands fields.tmp2 to the Jacobian as output and scratch at once,
    src/timestep.jl:159; default False: the conservative Jacobian),
    ``ma_bc_guess`` (correct each predicted guess for the current surface
    buoyancy with one exact per-mode vertical solve; default True),
    ``nmembers`` (independent ensemble members on this grid with these
    parameters, advanced together: every kernel pass covers all members in
    one launch; fields gain a last axis of length nmembers, set_b_ takes
    (Nx, Ny, nmembers), and each member's fields equal those of a
    one-member problem bit for bit; surface diagnostics and the adjoint need
    one member), ``device``.
    """

    def __init__(self, domain, *, scheme=RK3, dt=0.01, initial_time=0.0, adaptive_dt=False, filter_freq=10,
                 filter_strength=0.1, enable_diagnostics=True, output_dir="output", eps=0.01, ma_tol=1e-10,
                 ma_maxiter=50, ma_per_stage=True, ma_rhs="surface", ma_predictor="auto", filter_order=4,
                 filter_cutoff=0.65, filter=None, precision="fp64", ab2_literal_alias=False, ma_bc_guess=True,
                 nmembers=1, autotune=False, device=0):
        self.domain = domain
        self.timestepper = TimeParams(dt, scheme=scheme, adaptive_dt=adaptive_dt, filter_freq=filter_freq,
                                      filter_strength=filter_strength)
        cfg = _lib.default_config()
        cfg.nx, cfg.ny, cfg.nz = domain.Nx, domain.Ny, domain.Nz
        cfg.lx, cfg.ly, cfg.lz = domain.Lx, domain.Ly, domain.Lz
        cfg.eps = float(eps)
        cfg.dt = float(dt)
        cfg.scheme = _SCHEMES[scheme]
        cfg.filter_freq = int(filter_freq)
        cfg.filter_order = int(filter_order)
        cfg.filter_strength = float(filter_strength)
        cfg.filter_cutoff = float(filter_cutoff)
        cfg.ma_tol = float(ma_tol)
        cfg.ma_maxiter = int(ma_maxiter)
        cfg.ma_per_stage = 1 if ma_per_stage else 0
        cfg.ma_rhs_mode = {"surface": _lib.MA_RHS_SURFACE, "volume": _lib.MA_RHS_VOLUME}[ma_rhs]
        if ma_predictor == "auto":
            # measured at 1024^2 x 32 over steps 100-1000 with the boundary-
            # corrected guess: cubic in FP64 (1.91 iterations per step);
            # quadratic in mixed precision (1.23 per step, 3.6e-7 to 6.3e-7
            # error after 1000 steps on three initial fields).  The linear
            # guess takes 1.03-1.11 per step but its solves, stopped at the
            # first iteration, leave 1.5e-6 after 1000 steps on the k0 = 24
            # field; cubic takes 1.94 (the history is converged only to the
            # FP32 floor, and higher orders amplify its error)
            ma_predictor = "quadratic" if precision == "mixed" else "cubic"
        cfg.ma_predictor = {"previous": 0, "extrapolate": 1, "quadratic": 2, "cubic": 3}[ma_predictor]
        cfg.precision = {"fp64": 0, "mixed": 1}[precision]
        cfg.ab2_literal_alias = 1 if ab2_literal_alias else 0
        cfg.ma_bc_guess = 1 if ma_bc_guess else 0
        cfg.nmembers = int(nmembers)
        if cfg.nmembers > 1:
            enable_diagnostics = False  # surface diagnostics are per one-member problem
        from . import filter as _flt
        if filter is not None:
            if isinstance(filter, _flt.ExponentialFilter):
                cfg.filter_type = _lib.FILTER_EXPONENTIAL
                cfg.filter_strength, cfg.filter_order, cfg.filter_cutoff = filter.strength, filter.order, filter.cutoff
            elif isinstance(filter, _flt.HyperviscosityFilter):
                cfg.filter_type = _lib.FILTER_HYPERVISCOSITY
                cfg.filter_strength, cfg.filter_order = filter.coefficient, filter.order
            elif isinstance(filter, _flt.CutoffFilter):
                cfg.filter_type, cfg.filter_cutoff = _lib.FILTER_CUTOFF, filter.cutoff
            elif isinstance(filter, _flt.CesaroFilter):
                cfg.filter_type, cfg.filter_cutoff, cfg.filter_order = _lib.FILTER_CESARO, filter.cutoff, filter.order
        self._ctx = _Context(cfg, device)
        self.filter = filter
        if domain.z_grid != "uniform":
            dz = np.ascontiguousarray(domain.dz, dtype=np.float64)
            check(load().ssg_set_vertical_grid(self._ctx.h, dz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               dz.size), self._ctx.h)
        if filter is not None and isinstance(filter, _flt.CustomFilter):
            install_filter_(self, filter)
        self._ctx.set_time(float(initial_time), 0)
        if autotune:
            self._ctx.autotune()
        self.fields = Fields(self._ctx, domain)
        self.clock = TimeState(self._ctx, self.fields)
        self.diagnostics = DiagnosticTimeSeries() if enable_diagnostics else None
        self.output_settings = dict(dir=output_dir, save_freq=100, diag_freq=10, verbose=False)
        self.last_ma = None

    @property
    def eps(self):
        return self._ctx.cfg.eps

    @property
    def tiles(self):
        """Block shapes (threads per block) of the row and column-pair
        transform passes; (0, 0) is the built-in default."""
        return self._ctx.tiles()

    @property
    def variants(self):
        """(y_pass, thomas_staged): the Monge-Ampere y-pass kernel (0 plain
        loads, 1 TMA tiles, 2/4/8 one warp per transform with that many warps
        per block) and the vertical-solve form (1 staged through shared
        memory)."""
        return self._ctx.variants()

    def autotune(self, reps=3):
        """Time the candidate block shapes on this problem's grid and keep the
        fastest (ssg_autotune); the state is left as it was."""
        return self._ctx.autotune(reps)

    def close(self):
        self._ctx.close()


def set_b_(prob, b, domain=None):
    """set_b! (src/setICs.jl:21-88): zero mean, dealias, Monge-Ampere solve.
    Returns the solve's (iterations, converged, update)."""
    st = prob._ctx.set_b(b)
    prob.last_ma = (st.iterations, bool(st.converged), st.update)
    if prob.diagnostics is not None:
        update_diagnostics_(prob.diagnostics, prob.fields, prob.domain, prob.clock)
    return prob.last_ma


def solve_monge_ampere_fields_(fields_or_prob, domain=None, *, tol=None, verbose=False, eps=None):
    """solve_monge_ampere_fields! (src/poisson.jl:1068-1090): returns converged.
    ``tol`` and ``eps`` are fixed when the problem is created; passing other
    values raises."""
    ctx = fields_or_prob._ctx
    if tol is not None and tol != ctx.cfg.ma_tol:
        raise ValueError("tol is fixed at problem creation (ma_tol)")
    if eps is not None and eps != ctx.cfg.eps:
        raise ValueError("eps is fixed at problem creation")
    st = ctx.solve_ma()
    if verbose:
        print(f"[SSG] {st.iterations} iterations, update {st.update:.3e}")
    return bool(st.converged)


def timestep_(fields_or_prob, domain=None, params=None, state=None):
    """timestep! (src/timestep.jl:267-285): one step, returns dt."""
    ctx = fields_or_prob._ctx
    dt = params.dt if params is not None else ctx.cfg.dt
    if params is not None and _SCHEMES[params.scheme] != ctx.cfg.scheme:
        raise ValueError("the scheme is fixed at problem creation")
    ctx.step(1, dt)
    return dt


def step_until_(prob, stop_time, timestepper=None):
    """step_until! (src/timestep.jl:404-444): the last step is shortened to
    land on stop_time."""
    ts = timestepper or prob.timestepper
    t = prob.clock.t
    if not stop_time > t:
        raise ValueError(f"stop_time ({stop_time}) must be greater than current time ({t})")
    while t < stop_time:
        dt_use = min(ts.dt, stop_time - t)
        prob._ctx.step(1, dt_use)
        if prob.diagnostics is not None:
            update_diagnostics_(prob.diagnostics, prob.fields, prob.domain, prob.clock)
        t = prob.clock.t
    prob._ctx.set_time(float(stop_time), prob.clock.step)


def stepforward_(prob, nsteps=1, *, preserve_timestepper=False, custom_timestepper=None):
    """stepforward! (src/timestep.jl:449-482)."""
    ts = custom_timestepper or prob.timestepper
    if prob.diagnostics is None:
        return prob._ctx.step(nsteps, ts.dt)
    st = None
    for _ in range(int(nsteps)):
        st = prob._ctx.step(1, ts.dt)
        if prob.clock.step % prob.output_settings["diag_freq"] == 0:
            update_diagnostics_(prob.diagnostics, prob.fields, prob.domain, prob.clock)
    return st


def install_filter_(prob, filt, dt=None):
    """Make ``filt`` the problem's filter (any src/filter.jl type), as a
    transfer table on the dealiased modes."""
    from .filter import transfer_table
    tab = transfer_table(prob.domain, filt, dt if dt is not None else prob._ctx.cfg.dt)
    _install_table(prob, tab)
    prob.filter = filt


def _install_table(prob, tab):
    tab = np.asfortranarray(np.asarray(tab, dtype=np.float64))
    rc = load().ssg_set_filter_table(prob._ctx.h, tab.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), tab.size)
    check(rc, prob._ctx.h)
    # the device's filter is now this table (SSG_FILTER_CUSTOM)
    prob._ctx.cfg.filter_type = _lib.FILTER_CUSTOM
    prob._ctx.filter_table = tab


def apply_spectral_filter_(prob, domain=None, filt=None, dt=None):
    """apply_spectral_filter! (src/timestep.jl:247-260, src/filter.jl:181-192):
    filter the surface buoyancy once.  With ``filt`` (a filter object or, as
    the reference's legacy form, a strength for ExponentialFilter(strength,
    4, 0.65)) that filter becomes the problem's filter first."""
    from . import filter as _flt
    if filt is not None:
        if not isinstance(filt, _flt.AbstractSpectralFilter):
            filt = _flt.ExponentialFilter(float(filt), 4, 0.65)
        install_filter_(prob, filt, dt)
    check(load().ssg_apply_filter(prob._ctx.h), prob._ctx.h)


_CKPT_CONFIG_FIELDS = ("nx", "ny", "nz", "lx", "ly", "lz", "eps", "dt", "scheme", "filter_freq", "filter_order",
                       "ma_maxiter", "filter_strength", "filter_cutoff", "ma_tol", "ma_per_stage", "ma_rhs_mode",
                       "precision", "ma_predictor", "filter_type", "ab2_literal_alias", "ma_bc_guess")
_SCHEME_NAMES = {_lib.SCHEME_AB2: AB2_LowStorage, _lib.SCHEME_RK3: RK3}


def _rfft2(a):
    """rfft_2d! of (nx, ny[, nz]) real arrays: (nx, ny//2+1[, nz]) complex."""
    return np.fft.rfft2(a, axes=(0, 1))


def _geostrophic_3d(phi, domain):
    """u = -dPhi/dy, v = dPhi/dx on every level (spectral derivatives)."""
    ph = _rfft2(phi)
    kx = domain.kx[:, None, None]
    ky = domain.ky[None, :, None]
    u = -np.fft.irfft2(1j * ky * ph, s=phi.shape[:2], axes=(0, 1))
    v = np.fft.irfft2(1j * kx * ph, s=phi.shape[:2], axes=(0, 1))
    return np.asfortranarray(u), np.asfortranarray(v)


def save_simulation_state_full(filename, prob, *, save_spectral=True, save_diagnostics=True, save_metadata=True,
                               compress=True):
    """save_simulation_state_full(filename, prob) (src/output.jl:318-448).

    Writes the reference's datasets under its key paths -- ``time``, ``step``,
    ``dt``, ``grid/{Nx,Ny,Nz,Lx,Ly,Lz,x,y,z,dz,kx,ky}``,
    ``fields/surface/{buoyancy,streamfunction}``,
    ``fields/3d/{streamfunction,u_velocity,v_velocity}`` (u, v: the
    geostrophic velocities of Phi on every level),
    ``fields/spectral/{2d,3d}/*_{real,imag}`` (rfft_2d! layout, Nx x Ny/2+1),
    ``timestepper/*``, ``diagnostics/*``, ``metadata/*`` -- plus
    ``timestepper/db_dt_old`` (the AB2 history the reference does not save)
    and, under ``ssg_b200/``, the device state blob, the configuration, the
    vertical grid and a custom filter table, from which
    load_simulation_state_full continues the run bit for bit.

    The reference writes JLD2 (HDF5); this writes an .npz archive with the
    same key paths (h5py is not available here).  For compatibility with an
    earlier form of this function, ``(prob, filename)`` is accepted too."""
    if isinstance(filename, SemiGeostrophicProblem):
        filename, prob = prob, filename
    filename = str(filename)
    ctx = prob._ctx
    if ctx.members > 1:
        raise ValueError("save_simulation_state_full: one member per file (this problem holds "
                         f"{ctx.members}); _ctx.checkpoint() keeps every member's exact state")
    dom = prob.domain
    blob = ctx.checkpoint()
    t, step = ctx.time()
    ts = prob.timestepper
    bs, phis, phi = prob.fields.bs, prob.fields.phis, prob.fields.phi
    out = {
        "time": np.float64(t), "step": np.int64(step), "dt": np.float64(ts.dt),
        "grid/Nx": np.int64(dom.Nx), "grid/Ny": np.int64(dom.Ny), "grid/Nz": np.int64(dom.Nz),
        "grid/Lx": np.float64(dom.Lx), "grid/Ly": np.float64(dom.Ly), "grid/Lz": np.float64(dom.Lz),
        "grid/x": dom.x, "grid/y": dom.y, "grid/z": np.asarray(dom.z, dtype=np.float64),
        "grid/dz": np.asarray(dom.dz, dtype=np.float64),
        "fields/surface/buoyancy": bs, "fields/surface/streamfunction": phis,
        "fields/3d/streamfunction": phi,
        "timestepper/scheme": np.array(ts.scheme), "timestepper/dt": np.float64(ts.dt),
        "timestepper/adaptive_dt": np.bool_(ts.adaptive_dt), "timestepper/filter_freq": np.int64(ts.filter_freq),
        "timestepper/filter_strength": np.float64(ts.filter_strength),
        "timestepper/cfl_safety": np.float64(ts.cfl_safety), "timestepper/max_dt": np.float64(ts.max_dt),
        "timestepper/min_dt": np.float64(ts.min_dt),
        "timestepper/db_dt_old": prob.clock.db_dt_old,
    }
    u3, v3 = _geostrophic_3d(phi, dom)
    out["fields/3d/u_velocity"], out["fields/3d/v_velocity"] = u3, v3
    if save_spectral:
        out["grid/kx"], out["grid/ky"] = np.asarray(dom.kx), np.asarray(dom.ky)
        for name, f in (("2d/buoyancy", _rfft2(bs)), ("2d/streamfunction", _rfft2(phis)),
                        ("3d/streamfunction", _rfft2(phi))):
            out[f"fields/spectral/{name}_real"] = np.asfortranarray(f.real)
            out[f"fields/spectral/{name}_imag"] = np.asfortranarray(f.imag)
    diag = prob.diagnostics
    if save_diagnostics and diag is not None and len(diag.times) > 0:
        for k in ("times", "kinetic_energy", "enstrophy", "total_buoyancy", "max_divergence", "max_cfl"):
            out[f"diagnostics/{k}"] = np.asarray(getattr(diag, k), dtype=np.float64)
    if save_metadata:
        import datetime
        import socket
        dzs = np.abs(np.asarray(dom.dz))
        out.update({
            "metadata/creation_time": np.array(datetime.datetime.now().isoformat()),
            "metadata/hostname": np.array(socket.gethostname()), "metadata/mpi_size": np.int64(1),
            "metadata/precision": np.array({0: "Float64", 1: "Float64 (FP32 Monge-Ampere transforms)"}[
                ctx.cfg.precision]),
            "metadata/equation_type": np.array("surface_semi_geostrophic"),
            "metadata/description": np.array("Surface buoyancy evolution with Monge-Ampere constraint"),
            "metadata/file_type": np.array("complete_simulation_state"),
            "metadata/has_spectral_data": np.bool_(save_spectral),
            "metadata/has_diagnostics": np.bool_(save_diagnostics and diag is not None),
            "metadata/physics/domain_aspect_ratio": np.float64(dom.Lx / dom.Ly),
            "metadata/physics/grid_spacing_x": np.float64(dom.Lx / dom.Nx),
            "metadata/physics/grid_spacing_y": np.float64(dom.Ly / dom.Ny),
            "metadata/physics/grid_spacing_z_min": np.float64(dzs.min()),
            "metadata/physics/grid_spacing_z_max": np.float64(dzs.max()),
            "metadata/physics/z_boundary": np.array(str(dom.z_boundary)),
            "metadata/physics/z_grid": np.array(str(dom.z_grid)),
        })
    # the exact device state and what rebuilds its context
    cfg = {f: getattr(ctx.cfg, f) for f in _CKPT_CONFIG_FIELDS}
    sp = None
    if dom.stretch_params is not None:
        sp = {k: ([float(x) for x in np.ravel(v)] if k == "z_coords" else v) for k, v in dom.stretch_params.items()}
    out["ssg_b200/state"] = blob
    out["ssg_b200/config"] = np.array(repr(cfg))
    out["ssg_b200/grid"] = np.array(repr({"z_grid": dom.z_grid, "stretch_params": sp}))
    table = getattr(ctx, "filter_table", None)
    if cfg["filter_type"] == _lib.FILTER_CUSTOM and table is not None:
        out["ssg_b200/filter_table"] = table
    (np.savez_compressed if compress else np.savez)(filename, **out)
    # np.savez appends .npz to a name without it
    return filename if filename.endswith(".npz") else filename + ".npz"


def _filter_from_config(cfg):
    from . import filter as _flt
    ft = cfg["filter_type"]
    if ft == _lib.FILTER_HYPERVISCOSITY:
        return _flt.HyperviscosityFilter(cfg["filter_strength"], cfg["filter_order"])
    if ft == _lib.FILTER_CUTOFF:
        return _flt.CutoffFilter(cfg["filter_cutoff"])
    if ft == _lib.FILTER_CESARO:
        return _flt.CesaroFilter(cfg["filter_cutoff"], cfg["filter_order"])
    return None  # exponential: from the keyword parameters; custom: the saved table


def load_simulation_state_full(filename, domain=None, *, load_spectral=True, load_diagnostics=True,
                               validate_grid=True, device=0):
    """load_simulation_state_full(filename, domain) (src/output.jl:1011-1125):
    a new problem holding the saved state.  Returns the problem.

    A file written by save_simulation_state_full above carries the device
    state blob: the problem is rebuilt with the saved configuration (scheme,
    filter -- a custom table included --, solver settings, vertical grid) and
    continues bit for bit.  A file with only the reference's datasets is read
    the way the reference reads it: a problem from ``timestepper/*`` (scheme,
    dt, filter cadence and strength), the clock from ``time``/``step``, the
    surface buoyancy from ``fields/surface/buoyancy`` and, when present, the
    AB2 history from ``timestepper/db_dt_old``; the potential is then solved
    from that buoyancy (the stored one is its solution).  ``domain`` may be
    omitted; it is then rebuilt from ``grid/*``.  With ``validate_grid`` a
    domain of another shape raises, as in the reference."""
    import ast
    filename = str(filename)
    with np.load(filename, allow_pickle=False) as z:
        keys = set(z.files)
        get = lambda k: z[k][()] if z[k].shape == () else np.asarray(z[k])
        nx, ny, nz = int(get("grid/Nx")), int(get("grid/Ny")), int(get("grid/Nz"))
        lx, ly, lz = float(get("grid/Lx")), float(get("grid/Ly")), float(get("grid/Lz"))
        if domain is not None and validate_grid:
            ok = (nx, ny, nz) == (domain.Nx, domain.Ny, domain.Nz) and all(
                math.isclose(a, b, rel_tol=1e-10) for a, b in ((lx, domain.Lx), (ly, domain.Ly), (lz, domain.Lz)))
            if not ok:
                raise ValueError(f"Grid incompatibility detected!\nFile: {nx}x{ny}x{nz}, Lx={lx}, Ly={ly}, Lz={lz}\n"
                                 f"Domain: {domain.Nx}x{domain.Ny}x{domain.Nz}, Lx={domain.Lx}, Ly={domain.Ly}, "
                                 f"Lz={domain.Lz}")
        t, step = float(get("time")), int(get("step"))
        scheme = str(get("timestepper/scheme"))
        diag = {}
        if load_diagnostics and "diagnostics/times" in keys:
            for k in ("times", "kinetic_energy", "enstrophy", "total_buoyancy", "max_divergence", "max_cfl"):
                diag[k] = [float(x) for x in np.asarray(z[f"diagnostics/{k}"])]
        if "ssg_b200/state" in keys:
            blob = np.ascontiguousarray(z["ssg_b200/state"])
            cfg = ast.literal_eval(str(get("ssg_b200/config")))
            grid = ast.literal_eval(str(get("ssg_b200/grid")))
            table = np.asarray(z["ssg_b200/filter_table"]) if "ssg_b200/filter_table" in keys else None
            if domain is None:
                domain = make_domain(nx, ny, nz, Lx=lx, Ly=ly, Lz=lz, z_grid=grid["z_grid"],
                                     stretch_params=grid["stretch_params"])
            filt = _filter_from_config(cfg)
            prob = SemiGeostrophicProblem(
                domain, scheme=_SCHEME_NAMES[cfg["scheme"]], dt=cfg["dt"], eps=cfg["eps"],
                filter_freq=cfg["filter_freq"], filter_strength=cfg["filter_strength"], ma_tol=cfg["ma_tol"],
                ma_maxiter=cfg["ma_maxiter"], ma_per_stage=bool(cfg["ma_per_stage"]),
                ma_rhs=("surface", "volume")[cfg["ma_rhs_mode"]],
                ma_predictor=("previous", "extrapolate", "quadratic", "cubic")[cfg["ma_predictor"]],
                filter_order=cfg["filter_order"], filter_cutoff=cfg["filter_cutoff"], filter=filt,
                precision=("fp64", "mixed")[cfg["precision"]],
                ab2_literal_alias=bool(cfg.get("ab2_literal_alias", 0)), ma_bc_guess=bool(cfg.get("ma_bc_guess", 1)),
                enable_diagnostics=load_diagnostics, device=device)
            if cfg["filter_type"] == _lib.FILTER_CUSTOM:
                if table is None:
                    raise ValueError("checkpoint: custom filter without its transfer table")
                _install_table(prob, table)
            prob._ctx.restore(blob)
        else:
            if domain is None:
                domain = make_domain(nx, ny, nz, Lx=lx, Ly=ly, Lz=lz)
                if "grid/dz" in keys and not np.allclose(np.asarray(z["grid/dz"]), domain.dz, rtol=1e-14, atol=0):
                    domain = make_domain(nx, ny, nz, Lx=lx, Ly=ly, Lz=lz, z_grid="custom",
                                         stretch_params={"z_coords": np.asarray(z["grid/z"])})
            prob = SemiGeostrophicProblem(
                domain, scheme=scheme, dt=float(get("timestepper/dt")),
                filter_freq=int(get("timestepper/filter_freq")),
                filter_strength=float(get("timestepper/filter_strength")), enable_diagnostics=load_diagnostics,
                device=device)
            prob.fields.bs = np.asarray(z["fields/surface/buoyancy"], dtype=np.float64)
            if "timestepper/db_dt_old" in keys:
                prob.clock.db_dt_old = np.asarray(z["timestepper/db_dt_old"], dtype=np.float64)
            prob._ctx.set_time(t, step)
            prob._ctx.solve_ma()
    if diag and prob.diagnostics is not None:
        for k, v in diag.items():
            setattr(prob.diagnostics, k, v)
    return prob


def compute_surface_geostrophic_velocities_(fields, domain=None):
    """compute_surface_geostrophic_velocities! (src/setICs.jl:161-192):
    returns (u, v) at the surface."""
    return fields.u, fields.v
