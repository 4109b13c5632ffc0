"""Ensemble sharding and gathering (the multi-GPU form of the path: members are
independent, so ranks share no data-path collective).  The multi-rank logic
runs here as world_size-2 gloo process groups on CPU, with oracle members
standing in for the GPU ones."""
import os
import pickle
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

CONFIG5 = [(128, 128, 16)] * 64 + [(256, 256, 16)] * 16


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_shard_members_balanced_and_complete(ssg, world):
    from ssg_b200.ensemble import member_cost, shard_members
    parts = shard_members(CONFIG5, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(CONFIG5)))
    loads = [sum(member_cost(*CONFIG5[i]) for i in p) for p in parts]
    assert max(loads) / (sum(loads) / world) < 1.05


class OracleMember:
    """CPU stand-in for a GPU member (test only)."""

    def __init__(self, i, grids):
        import oracle
        nx, ny, nz = grids[i]
        self.o = oracle.Oracle(nx, ny, nz, dt=1e-3, eps=0.01, filter_order=8)
        import ssg_b200
        self.o.set_b(ssg_b200.ic.perturbed_member(nx, ny, 4, 7, i))

    def step(self, n):
        self.o.step(n)

    def result(self):
        import oracle
        return {"bs": self.o.get(oracle.FIELD_B_S), "t": self.o.time()[0]}


GRIDS = [(32, 32, 6), (64, 64, 6), (32, 32, 6), (32, 32, 6), (64, 64, 6)]


def _worker(rank, world, port, out_path):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path.insert(0, os.path.join(root, "ssg.jl_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    sys.path.insert(0, here)
    import torch.distributed as dist
    from datetime import timedelta
    from ssg_b200.ensemble import Ensemble
    from test_ensemble import GRIDS, OracleMember
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    ens = Ensemble(GRIDS, lambda i: OracleMember(i, GRIDS), rank=rank, world_size=world, max_threads=2)
    ens.step(3)
    res = ens.gather(dist)
    if rank == 0:
        with open(out_path, "wb") as f:
            pickle.dump({"res": res, "owned": ens.owned}, f)
    ens.close()
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_ensemble_gather_matches_single_process(ssg, oracle_mod, tmp_path):
    from ssg_b200.ensemble import Ensemble
    out = str(tmp_path / "res.pkl")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    with open(out, "rb") as f:
        got = pickle.load(f)["res"]
    single = Ensemble(GRIDS, lambda i: OracleMember(i, GRIDS))
    single.step(3)
    ref = single.gather()
    single.close()
    assert len(got) == len(GRIDS)
    for a, b in zip(got, ref):
        assert a["t"] == b["t"]
        assert np.array_equal(a["bs"], b["bs"])


@pytest.mark.gpu
@pytest.mark.parametrize("batched,mode", [(False, None), (True, "threads"), (True, "one_graph")])
def test_concurrent_gpu_members_match_solo_runs(require_gpu, ssg, batched, mode):
    """Members stepped together (host threads, or one CUDA graph launch per
    chunk) give bit for bit the fields of solo runs."""
    from ssg_b200.ensemble import Ensemble, GPUMember
    grids = [(64, 64, 8), (128, 128, 8), (64, 64, 8), (128, 128, 8)]
    fields = [ssg.ic.perturbed_member(g[0], g[1], 5, 3, m) for m, g in enumerate(grids)]

    def make(i):
        nx, ny, nz = grids[i]
        dom = ssg.make_domain(nx, ny, nz)
        p = ssg.SemiGeostrophicProblem(dom, scheme=ssg.AB2_LowStorage, dt=1e-3, filter_order=8,
                                       enable_diagnostics=False)
        ssg.set_b_(p, fields[i], dom)
        return GPUMember(p)

    ens = Ensemble(grids, make, max_threads=4, batched=batched, batch_mode=mode or "threads")
    ens.step(6)
    ens.step(7)
    together = ens.gather()
    ens.close()
    for i in range(len(grids)):
        m = make(i)
        m.step(13)
        solo = m.result()
        m.close()
        assert np.array_equal(solo["bs"], together[i]["bs"])
