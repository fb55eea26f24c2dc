"""Multi-rank replica path on CPU: two gloo ranks split a batch of
independent instances, solve their shards with the CPU oracle, gather, and
reproduce the serial result; timing uses the max over ranks."""

import os
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _instances():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from cases import QED_CASES

    names = ["qed2d_3x2_q0", "qed2d_3x2_Q-2", "qed2d_3x2_Q-1", "qed2d_3x2_Q+1", "qed2d_3x2_Q+2", "qed1d_L8_obc"]
    return [(n, QED_CASES[n]) for n in names]


def _solve(name):
    from cases import build
    from oracle import edlgt_oracle as O

    model, g, m = build(name)
    cfg = O.sector_configs(**model.sector_inputs)
    H = O.assemble(model.hamiltonian_blocks(g, m), cfg, model.loc_dims)
    w, _ = O.lowest_eigs(H, 1)
    return len(cfg), float(w[0])


def _worker(rank, world, port, q):
    import torch.distributed as dist

    for p in (os.path.join(ROOT, "ed-lgt_b200"), ROOT, os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from edgpu.replicas import gather_objects, max_over_ranks, shard_instances

    inst = _instances()
    dims = [_solve(n)[0] for n, _ in inst]  # cost proxy: dimension
    mine = shard_instances(dims, world, rank)
    res = {i: _solve(inst[i][0])[1] for i in mine}
    allres = gather_objects(res, world)
    tmax = max_over_ranks(float(rank + 1), world)
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        merged = {}
        for r in allres:
            merged.update(r)
        q.put((merged, tmax, [shard_instances(dims, world, r) for r in range(world)]))


@pytest.mark.timeout(300)
def test_two_rank_shards_reproduce_serial():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged, tmax, shards = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    inst = _instances()
    assert sorted(merged) == list(range(len(inst)))
    assert sorted(shards[0] + shards[1]) == list(range(len(inst))) and not set(shards[0]) & set(shards[1])
    for i, (name, _) in enumerate(inst):
        assert abs(merged[i] - _solve(name)[1]) < 1e-12
    assert tmax == 2.0


def test_shard_balance_is_deterministic():
    from edgpu.replicas import shard_instances

    costs = [90, 26, 52, 67, 26, 90, 90, 10]
    a = [shard_instances(costs, 3, r) for r in range(3)]
    b = [shard_instances(costs, 3, r) for r in range(3)]
    assert a == b
    assert sorted(sum(a, [])) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in a]
    assert max(loads) - min(loads) <= max(costs)
