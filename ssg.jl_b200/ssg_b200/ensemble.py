"""Ensembles of independent SSG problems (perturbed members, uneven grids).

Members never exchange data, so an ensemble shards by member: each rank (one
process per GPU) owns a work-balanced subset, steps it with no collective,
and the per-member results are gathered to rank 0 at the end.  On one GPU the
members of a rank advance concurrently, in one of two ways:
  - batched (``DeviceBatch``, libssg_b200's ssg_ensemble_*): one CUDA graph
    launch advances every member by a chunk of steps, each member's steps an
    independent branch of the graph;
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
    mode "one_graph" (default): one CUDA graph launch per chunk of steps
    advances all members; mode "threads": each member steps as in ssg_step
    (cached CUDA graphs on its own stream), library worker threads issuing the
    launches in parallel.  On the 80-member 128^2/256^2 workload the one-graph
    form measured 1176-1252 ensemble steps/s, the threaded form 699-1239 (it
    varies with how the host threads are scheduled).  With ``autotune``, the block shapes and kernel variants of each
    distinct member grid are tuned once (ssg_autotune) and shared by the
    members of that grid; ``tiles`` maps (nx, ny, nz, precision) to the chosen
    (x_threads, y_threads) and ``variants`` to the chosen (y_pass,
    thomas_staged)."""

    MODES = {"threads": 0, "one_graph": 1}

    def __init__(self, probs, mode="one_graph", autotune=False):
        from ._lib import check, load
        self.probs = list(probs)
        self.tiles = {}
        self.variants = {}
        if autotune:
            # one tuning per distinct (grid, precision); members of the same
            # kind share its block shapes and kernel variants
            for p in self.probs:
                c = p._ctx.cfg
                key = (c.nx, c.ny, c.nz, c.precision)
                if key not in self.tiles:
                    self.tiles[key] = p._ctx.autotune()
                    self.variants[key] = p._ctx.variants()
                else:
                    p._ctx.set_tiles(*self.tiles[key])
                    p._ctx.set_variants(*self.variants[key])
        L = load()
        arr = (ctypes.c_void_p * len(self.probs))(*[p._ctx.h.value for p in self.probs])
        self.h = ctypes.c_void_p()
        check(L.ssg_ensemble_create(arr, len(self.probs), self.MODES[mode], ctypes.byref(self.h)), None)

    def step(self, n):
        from ._lib import SsgError, SsgStepStats, load
        L = load()
        stats = (SsgStepStats * len(self.probs))()
        rc = L.ssg_ensemble_step(self.h, int(n), stats)
        if rc != 0:
            msg = L.ssg_ensemble_last_error(self.h)
            raise SsgError(rc, msg.decode() if msg else "")
        return list(stats)

    def close(self):
        from ._lib import load
        if self.h is not None and self.h.value:
            load().ssg_ensemble_destroy(self.h)
        self.h = None


class Ensemble:
    """Members owned by this rank, stepped concurrently.

    ``make_member(i)`` returns an object with ``step(n)`` and ``result()``
    (for a GPU member: a SemiGeostrophicProblem wrapped by ``GPUMember``).
    With ``batched`` (and GPU members), the rank's members advance as one
    DeviceBatch (``batch_mode`` "threads" or "one_graph", ``autotune`` as
    there); otherwise one Python host thread per member.
    """

    def __init__(self, grids, make_member, rank=0, world_size=1, max_threads=16, batched=False,
                 batch_mode="one_graph", autotune=False):
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
