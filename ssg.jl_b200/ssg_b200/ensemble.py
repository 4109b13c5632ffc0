"""Ensembles of independent SSG problems (perturbed members, uneven grids).

Members never exchange data, so an ensemble shards by member: each rank (one
process per GPU) owns a work-balanced subset, steps it with no collective,
and the per-member results are gathered to rank 0 at the end.  On one GPU the
members of a rank advance concurrently, in one of two ways:
  - batched (``DeviceBatch``, libssg_b200's ssg_members_* and ssg_ensemble_*):
    members that share a grid and configuration become the members of one
    context, whose every kernel pass covers all of them in one launch, and
    one CUDA graph launch advances every such context by a chunk of steps;
  - threaded: every member has its own context and CUDA stream, and one host
    thread per member drives it (the library calls release the GIL).
"""
import concurrent.futures as cf
import ctypes
import math

import numpy as np


def member_cost(nx, ny, nz):
    """Relative work of one member step: the transforms are O(N^2 log N) per
    plane, over nz planes."""
    return nx * ny * max(math.log2(nx * ny), 1.0) * nz


def shard_members(grids, world_size):
    """Assign members to ranks, balancing summed cost (largest first, each
    to the least-loaded rank).  Returns one sorted list of member indices per
    rank."""
    order = sorted(range(len(grids)), key=lambda i: -member_cost(*grids[i]))
    load = [0.0] * world_size
    owned = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        owned[r].append(i)
        load[r] += member_cost(*grids[i])
    return [sorted(o) for o in owned]


class DeviceBatch:
    """SemiGeostrophicProblems on one GPU advanced together (ssg_ensemble_step).

    mode "members" (default): problems that share a grid and configuration
    become the members of one context (ssg_config.nmembers, state moved over
    by ssg_members_gather), so every kernel pass covers all of them in one
    launch; the batched contexts (and any problem without a partner) then
    advance as one CUDA graph launch per chunk of steps.  The problems' own
    contexts hold their state again after ``sync()`` (called by ``close()``);
    each member's fields equal those of its problem stepped alone, bit for
    bit.  mode "one_graph": one CUDA graph launch per chunk of steps advances
    every problem's own context, each an independent branch; mode "threads":
    each problem steps as in ssg_step (cached CUDA graphs on its own stream),
    library worker threads issuing the launches in parallel.  With
    ``autotune``, the block shapes and kernel variants of each distinct
    context (grid, precision, members) are tuned once (ssg_autotune); ``tiles``
    maps (nx, ny, nz, precision) to the chosen (x_threads, y_threads) and
    ``variants`` to the chosen (y_pass, thomas_staged)."""

    MODES = {"threads": 0, "one_graph": 1, "members": 1}

    def __init__(self, probs, mode="members", autotune=False):
        from ._lib import check, load
        if mode not in self.MODES:
            raise ValueError(f"mode must be one of {sorted(self.MODES)}")
        self.probs = list(probs)
        self.mode = mode
        self.tiles = {}
        self.variants = {}
        self.groups = []  # (batched _Context, indices of its member problems)
        self._dirty = False
        ctxs = [p._ctx for p in self.probs]
        if mode == "members":
            ctxs = self._group()
        if autotune:
            # one tuning per distinct context kind; contexts of the same kind
            # share its block shapes and kernel variants
            tuned = {}
            for c in ctxs:
                cfg = c.cfg
                kind = (cfg.nx, cfg.ny, cfg.nz, cfg.precision, c.members)
                if kind not in tuned:
                    tuned[kind] = (c.autotune(), c.variants())
                else:
                    c.set_tiles(*tuned[kind][0])
                    c.set_variants(*tuned[kind][1])
                self.tiles.setdefault(kind[:4], tuned[kind][0])
                self.variants.setdefault(kind[:4], tuned[kind][1])
        self._ctxs = ctxs
        L = load()
        arr = (ctypes.c_void_p * len(ctxs))(*[c.h.value for c in ctxs])
        self.h = ctypes.c_void_p()
        check(L.ssg_ensemble_create(arr, len(ctxs), self.MODES[mode], ctypes.byref(self.h)), None)

    def _group(self):
        """Batched contexts for the problems that share a configuration,
        clock and tables; the contexts to step, in order."""
        from .api import _Context
        from ._lib import SsgError, check, load
        L = load()
        kinds = {}
        for i, p in enumerate(self.probs):
            c = p._ctx
            dom = p.domain
            table = getattr(c, "filter_table", None)
            key = (bytes(c.cfg), np.asarray(dom.dz, dtype=np.float64).tobytes(), c.time(),
                   None if table is None else np.asarray(table).tobytes(), getattr(c, "device", 0))
            kinds.setdefault(key, []).append(i)
        ctxs = []
        for key, idx in kinds.items():
            if len(idx) == 1:
                ctxs.append(self.probs[idx[0]]._ctx)
                continue
            src = self.probs[idx[0]]._ctx
            cfg = type(src.cfg).from_buffer_copy(src.cfg)
            cfg.nmembers = len(idx)
            bctx = _Context(cfg, getattr(src, "device", 0))
            solo = (ctypes.c_void_p * len(idx))(*[self.probs[i]._ctx.h.value for i in idx])
            try:
                check(L.ssg_members_gather(bctx.h, solo, len(idx)), bctx.h)
            except SsgError:
                # states that cannot share a context (predictor histories of
                # different lengths) step on their own
                bctx.close()
                ctxs.extend(self.probs[i]._ctx for i in idx)
                continue
            self.groups.append((bctx, idx))
            ctxs.append(bctx)
        return ctxs

    def step(self, n):
        """Advance every problem by n steps; one stats record per stepped
        context (a batched context's record sums its members' solves)."""
        from ._lib import SsgError, SsgStepStats, load
        L = load()
        stats = (SsgStepStats * len(self._ctxs))()
        rc = L.ssg_ensemble_step(self.h, int(n), stats)
        self._dirty = bool(self.groups)
        if rc != 0:
            msg = L.ssg_ensemble_last_error(self.h)
            raise SsgError(rc, msg.decode() if msg else "")
        return list(stats)

    def sync(self):
        """Copy the batched members' state back into the problems' own
        contexts (ssg_members_scatter)."""
        from ._lib import check, load
        if not self._dirty:
            return
        L = load()
        for bctx, idx in self.groups:
            solo = (ctypes.c_void_p * len(idx))(*[self.probs[i]._ctx.h.value for i in idx])
            check(L.ssg_members_scatter(bctx.h, solo, len(idx)), bctx.h)
        self._dirty = False

    def close(self):
        from ._lib import load
        if self.h is not None and self.h.value:
            load().ssg_ensemble_destroy(self.h)
        self.h = None
        if self.groups:
            try:
                self.sync()
            finally:
                for bctx, _ in self.groups:
                    bctx.close()
                self.groups = []


class Ensemble:
    """Members owned by this rank, stepped concurrently.

    ``make_member(i)`` returns an object with ``step(n)`` and ``result()``
    (for a GPU member: a SemiGeostrophicProblem wrapped by ``GPUMember``).
    With ``batched`` (and GPU members), the rank's members advance as one
    DeviceBatch (``batch_mode`` "members", "one_graph" or "threads",
    ``autotune`` as there); otherwise one Python host thread per member.
    """

    def __init__(self, grids, make_member, rank=0, world_size=1, max_threads=16, batched=False,
                 batch_mode="members", autotune=False):
        self.grids = list(grids)
        self.rank, self.world_size = rank, world_size
        self.owned = shard_members(self.grids, world_size)[rank]
        self.members = {i: make_member(i) for i in self.owned}
        self.pool = cf.ThreadPoolExecutor(max_workers=max(1, min(max_threads, len(self.owned))))
        self.batch = None
        if batched and self.owned and all(isinstance(self.members[i], GPUMember) for i in self.owned):
            self.batch = DeviceBatch([self.members[i].prob for i in self.owned], batch_mode, autotune=autotune)

    def step(self, n):
        if self.batch is not None:
            self.batch.step(n)
            return
        futs = [self.pool.submit(self.members[i].step, n) for i in self.owned]
        for f in futs:
            f.result()

    def results(self):
        if self.batch is not None:
            self.batch.sync()
        return {i: self.members[i].result() for i in self.owned}

    def gather(self, dist=None):
        """All members' results on rank 0, in member order (None elsewhere)."""
        mine = self.results()
        if dist is None or self.world_size == 1:
            return [mine[i] for i in range(len(self.grids))]
        parts = [None] * self.world_size
        dist.all_gather_object(parts, mine)
        if self.rank != 0:
            return None
        merged = {}
        for p in parts:
            merged.update(p)
        return [merged[i] for i in range(len(self.grids))]

    def close(self):
        if self.batch is not None:
            self.batch.close()
        self.pool.shutdown(wait=True)
        for m in self.members.values():
            close = getattr(m, "close", None)
            if close:
                close()


class GPUMember:
    """One SemiGeostrophicProblem as an ensemble member; result() returns its
    surface diagnostics and final buoyancy."""

    def __init__(self, prob, keep_field=True):
        self.prob = prob
        self.keep_field = keep_field

    def step(self, n):
        self.prob._ctx.step(n, self.prob._ctx.cfg.dt)

    def result(self):
        from .api import diagnostics
        out = diagnostics(self.prob)
        if self.keep_field:
            out["bs"] = self.prob.fields.bs
        return out

    def close(self):
        self.prob.close()


def perturbed_members(specs, k0, seed, amplitude=1e-3):
    """Initial fields of the ensemble workload: a seeded spectral-peak
    field plus an amplitude-scaled independent field of the same spectrum,
    one per member.  specs: list of (nx, ny)."""
    from .ic import perturbed_member
    return [perturbed_member(nx, ny, k0, seed, m, amplitude) for m, (nx, ny) in enumerate(specs)]
