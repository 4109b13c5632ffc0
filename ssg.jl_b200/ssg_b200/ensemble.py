"""Ensembles of independent SSG problems (perturbed members, uneven grids).

Members never exchange data, so an ensemble shards by member: each rank (one
process per GPU) owns a work-balanced subset, steps it with no collective,
and the per-member results are gathered to rank 0 at the end.  On one GPU the
members of a rank advance concurrently: every member has its own context and
CUDA stream, and one host thread per member drives it (the library calls
release the GIL), so kernels of different members overlap on the device.
"""
import concurrent.futures as cf
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


class Ensemble:
    """Members owned by this rank, stepped concurrently.

    ``make_member(i)`` returns an object with ``step(n)`` and ``result()``
    (for a GPU member: a SemiGeostrophicProblem wrapped by ``GPUMember``).
    """

    def __init__(self, grids, make_member, rank=0, world_size=1, max_threads=16):
        self.grids = list(grids)
        self.rank, self.world_size = rank, world_size
        self.owned = shard_members(self.grids, world_size)[rank]
        self.members = {i: make_member(i) for i in self.owned}
        self.pool = cf.ThreadPoolExecutor(max_workers=max(1, min(max_threads, len(self.owned))))

    def step(self, n):
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
