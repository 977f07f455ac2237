"""The multi-GPU path of bench.py is replicas: each rank runs its own
realisations and only the timing crosses ranks.  Checked here with two gloo
ranks on the CPU: distinct run seeds per rank, and every rank seeing the
slowest rank's time."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seen = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
        out.put((rank, bench.replica_seed(rank), seen))
    finally:
        dist.destroy_process_group()


def test_replica_ranks_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] != res[1][1]
    assert res[0][2] == res[1][2] == 20.0


def _gather_rank(rank, world, port, out):
    import numpy as np
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 7                                   # not a multiple of the ranks
        mine = bench.ensemble_share(n, rank, world)
        local = np.array([[100 * i + d for d in range(5)] for i in mine], float)
        full = bench.gather_series(local, n, rank, world, dist, "cpu")
        out.put((rank, mine, full.tolist()))
    finally:
        dist.destroy_process_group()


def test_ensemble_split_and_gather_over_gloo():
    """The C2 ensemble split by realisation across two ranks, and the all-gather of
    the members' daily series that ends the run."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    (r0, m0, f0), (r1, m1, f1) = res
    assert sorted(m0 + m1) == list(range(7)) and not set(m0) & set(m1)
    want = [[100 * i + d for d in range(5)] for i in range(7)]
    assert f0 == want and f1 == want
