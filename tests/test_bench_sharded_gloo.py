"""bench.py's uneven batch over two ranks (gloo on CPU): each rank steps its
own share of the runs, the whole-job value is the summed cell updates over
the slowest rank's device time, and a failure on one rank is reported
without leaving the other rank waiting in a collective. The batch itself is
replaced by a fake of autotune.batch_observables (no GPU here)."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, fail_rank, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from a5_streamer_b200 import autotune
        seen = []

        def fake(cfgs, schedule=None, **kw):
            seen.append(len(cfgs))
            if schedule is not None and rank == fail_rank:
                raise RuntimeError("planted failure")
            n = float(len(cfgs))
            return [], (1, 1000.0 * (rank + 1), 0.0, 1e6 * n), 2.0 * (rank + 1)

        autotune.batch_observables = fake
        out = bench.run_uneven_sharded(8, (0, 1, 1, 2, 2), rank, world, device=None)
        q.put((rank, out, seen))
    finally:
        dist.destroy_process_group()


def _run(fail_rank):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, fail_rank, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    return sorted((q.get(timeout=10) for _ in range(2)), key=lambda t: t[0])


def test_sharded_batch_sums_units_and_takes_the_slowest_rank():
    res = _run(fail_rank=-1)
    (r0, out0, seen0), (r1, out1, seen1) = res
    # every run on exactly one rank
    assert seen0[0] + seen1[0] == 8 and out0["runs_per_rank"] + out1["runs_per_rank"] == 8
    for out in (out0, out1):
        fp = out["fp64"]
        assert fp["cell_updates"] == 8e6
        assert fp["device_s_max_over_ranks"] == 2.0        # rank 1: 2000 ms
        assert fp["value"] == 8e6 / 2.0
        assert out["mixed"]["speedup_vs_fp64"] == 1.0


def test_a_failing_rank_is_reported_and_no_rank_hangs():
    res = _run(fail_rank=1)
    for _, out, _ in res:
        assert "value" in out["fp64"]
        assert "unavailable" in out["mixed"]
