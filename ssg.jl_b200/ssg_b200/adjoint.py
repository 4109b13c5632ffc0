"""Discrete adjoint of the time step (no counterpart in SSG.jl).

The gradient of a functional of the final surface buoyancy b_T with respect to
the initial buoyancy b0 handed to ``set_b_``, through ``nsteps`` steps of the
problem's scheme.  The forward run keeps a device checkpoint every
``ckpt_every`` steps; the reverse sweep recomputes each segment from its
checkpoint and runs the transposed steps backwards (libssg_b200's
``ssg_adjoint_record`` / ``ssg_adjoint``).

``rrule`` has the shape of ChainRulesCore's ``rrule``: it returns the primal
result and a pullback that maps a cotangent on b_T to one on b0.
"""
import ctypes

import numpy as np

from ._lib import SsgAdjointStats, check, load


def _as_field(a, ctx):
    a = np.asfortranarray(np.asarray(a, dtype=np.float64))
    if a.shape != (ctx.cfg.nx, ctx.cfg.ny):
        raise ValueError(f"expected shape {(ctx.cfg.nx, ctx.cfg.ny)}, got {a.shape}")
    return a


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _stats_dict(st):
    return {name: getattr(st, name) for name, _ in SsgAdjointStats._fields_}


def record_(prob, b0, nsteps, ckpt_every=20, t0=0.0):
    """Restart the clock at (t0, step 0), set_b_(prob, b0), then ``nsteps``
    steps with checkpoints kept on the device for ``adjoint``.  The problem
    ends at the final state."""
    ctx = prob._ctx
    a = _as_field(b0, ctx)
    ctx.set_time(t0, 0)
    st = SsgAdjointStats()
    rc = load().ssg_adjoint_record(ctx.h, _ptr(a), a.size, int(nsteps), int(ckpt_every), ctypes.byref(st))
    check(rc, ctx.h)
    return _stats_dict(st)


def adjoint(prob, dL_dbT):
    """(d b_T / d b0)^T dL_dbT for the run last recorded by ``record_``.
    Returns (dL_db0 as an (nx, ny) Fortran-ordered array, stats)."""
    ctx = prob._ctx
    g = _as_field(dL_dbT, ctx)
    out = np.zeros((ctx.cfg.nx, ctx.cfg.ny), dtype=np.float64, order="F")
    st = SsgAdjointStats()
    rc = load().ssg_adjoint(ctx.h, _ptr(g), _ptr(out), g.size, ctypes.byref(st))
    check(rc, ctx.h)
    return out, _stats_dict(st)


def rrule(prob, b0, nsteps, ckpt_every=20, t0=0.0):
    """Primal b_T = run(b0) and its pullback  dL/db_T -> dL/db0."""
    record_(prob, b0, nsteps, ckpt_every, t0)
    bT = prob.fields.bs

    def pullback(dL_dbT):
        return adjoint(prob, dL_dbT)[0]

    return bT, pullback


def misfit_loss_and_gradient(prob, b0, target, nsteps, ckpt_every=20, t0=0.0):
    """L = sum (b_T - target)^2 over the grid and dL/db0."""
    bT, pullback = rrule(prob, b0, nsteps, ckpt_every, t0)
    r = bT - np.asarray(target, dtype=np.float64)
    return float(np.sum(r * r)), pullback(2.0 * r)


def misfit_loss(prob, b0, target, nsteps, t0=0.0):
    """The same functional from a plain forward run (for finite differences):
    clock restarted at (t0, step 0), set_b_, ``nsteps`` steps."""
    from .api import set_b_
    ctx = prob._ctx
    ctx.set_time(t0, 0)
    set_b_(prob, b0, prob.domain)
    ctx.step(int(nsteps), ctx.cfg.dt)
    r = prob.fields.bs - np.asarray(target, dtype=np.float64)
    return float(np.sum(r * r))
