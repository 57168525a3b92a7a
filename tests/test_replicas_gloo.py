"""Multi-rank host logic on CPU with the gloo backend (world size 2):
max-over-ranks timing, whole-job throughput and the run partition."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from a5_streamer_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = 1.0 + rank  # rank 1 is the slow one
        m = replicas.max_over_ranks(t)
        units = replicas.sum_over_ranks(100.0 * (rank + 1))
        q.put((rank, m, units))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, m, units in res:
        assert m == 2.0 and units == 300.0
    assert replicas.replica_throughput(300.0, 2.0) == 150.0


def test_partition_is_balanced_and_complete():
    costs = [5, 1, 1, 1, 1, 1, 4, 2, 2]
    parts = replicas.partition_runs(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= 1
    assert replicas.partition_runs([], 2) == [[], []]
    with pytest.raises(ValueError):
        replicas.partition_runs([1], 0)
