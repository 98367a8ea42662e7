"""The N > 1 path on CPU: two gloo ranks run independent instances (the oracle
stands in for the GPU work), take the max of their times and the sum of their
counts, and shard a batch of instances by cost."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from crysscft_sample_b200 import replicas


def test_shard_instances_balanced_and_complete():
    costs = [64 ** 3 * 200, 16 ** 3 * 200, 48 ** 3 * 200, 32 ** 3 * 200, 24 ** 3 * 200] * 4
    for world in (1, 2, 3, 8):
        shards = replicas.shard_instances(costs, world)
        assert sorted(i for s in shards for i in s) == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(costs)
    assert replicas.shard_instances(costs, 2) == replicas.shard_instances(costs, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist = replicas.init(backend="gloo", timeout_s=60)
    from crysscft_sample_b200 import fields
    from oracle import scft_oracle as O

    costs = [16 ** 3, 8 ** 3, 16 ** 3, 8 ** 3]
    mine = replicas.shard_instances(costs, world)[rank]
    F = []
    for i in mine:
        n = 16 if costs[i] == 16 ** 3 else 8
        N = (2 * n,) * 3
        wA, wB = fields.seed_fields(N, 4.0, seed=100 + i)
        S = O.OracleSolver("PMMM", N)
        r = O.scft_iterations(S, 0.3, 0.02, 15.0, (4.0,) * 3, 0.1, 2,
                              fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB))
        F.append(r["F"][-1])
    replicas.barrier(dist)
    tmax = replicas.max_over_ranks(dist, float(rank + 1))
    count = replicas.sum_over_ranks(dist, float(len(mine)))
    out.put((rank, mine, F, tmax, count))
    dist.destroy_process_group()


def test_two_gloo_ranks_run_disjoint_instances():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert sorted(res[0][1] + res[1][1]) == [0, 1, 2, 3]
    assert all(r[3] == 2.0 for r in res)       # max over ranks
    assert all(r[4] == 4.0 for r in res)       # every instance counted once
    assert all(np.isfinite(f) for r in res for f in r[2])
