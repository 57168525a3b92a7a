"""Device-driven batch of independent runs (a5s_batch_run / a5g_batch_*):
uneven runs stepped together, the block's step sizes computed on the
device, the block replayed from a CUDA graph, regrids on host threads. Every
member must end bit-identical to the same run driven alone (a5s_run), which
the driver tests hold bit-identical to the oracle."""
import numpy as np
import pytest

from a5_streamer_b200 import config, streamer
from a5_streamer_b200.device import N_VAR_CELL

pytestmark = pytest.mark.gpu


def _members():
    runs = config.batch_cylindrical_runs(n=3, seed=7, end_time=1.0e-9)
    runs.append(config.cartesian_8mm(end_time=0.6e-9))
    runs.append(config.cylindrical_16mm(end_time=1.5e-9))
    return runs


def _same(a, b, where):
    ma, ga, la = a.tree.export()
    mb, gb, lb = b.tree.export()
    assert np.array_equal(ma, mb), f"{where}: topology differs"
    assert np.array_equal(ga, gb), f"{where}: geometry differs"
    for lvl in la:
        for x, y in zip(la[lvl], lb[lvl]):
            assert np.array_equal(x, y), f"{where}: level lists differ"
    assert a.time == b.time, (where, a.time, b.time)
    for iv in range(N_VAR_CELL):
        assert np.array_equal(a.device.cc(iv), b.device.cc(iv)), f"{where}: cell variable {iv}"
    for d in range(2):
        for f in range(2):
            assert np.array_equal(a.device.fc(d, f), b.device.fc(d, f)), f"{where}: face {d} {f}"


@pytest.mark.parametrize("use_graph,groups", [(False, 1), (True, 1), (True, 2)])
@pytest.mark.parametrize("mixed", [False, True])
def test_batch_equals_single_runs(use_graph, groups, mixed):
    cfgs = _members()
    sched = (0, 1, 1, 4, 1)
    batch = [streamer.Simulation(c) for c in cfgs]
    alone = [streamer.Simulation(c) for c in cfgs]
    for s in batch + alone:
        if mixed:
            s.device.set_precision(True, sched)
        s.init()
    nb, gpu_ms, host_ms, cu = streamer.run_batch(batch, [c.end_time for c in cfgs],
                                                 use_graph=use_graph, n_threads=4, groups=groups)
    assert nb > 0 and gpu_ms > 0 and cu > 0
    for k, (s, c) in enumerate(zip(alone, cfgs)):
        s.run(c.end_time)
        _same(batch[k], s, f"member {k}")


def test_batch_rejects_mixed_block_sizes():
    a = streamer.Simulation(config.cartesian_8mm())
    b = streamer.Simulation(config.cartesian_8mm(num_steps_amr=3))
    a.init()
    b.init()
    with pytest.raises(Exception):
        streamer.run_batch([a, b], 1e-10)


def test_batch_finished_runs_stay_put():
    """A member past its end time is skipped by every later block."""
    cfgs = [config.cartesian_8mm(end_time=0.2e-9), config.cartesian_8mm(end_time=0.8e-9)]
    sims = [streamer.Simulation(c) for c in cfgs]
    for s in sims:
        s.init()
    streamer.run_batch(sims, [c.end_time for c in cfgs])
    ref = streamer.Simulation(cfgs[0])
    ref.init()
    ref.run(cfgs[0].end_time)
    _same(sims[0], ref, "short member")
    assert sims[1].time > cfgs[1].end_time


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_with_blocks_per_run_equals_single_runs(use_graph):
    """Box-to-block mapping: members take 1, 3, 2, 4 and 1 blocks of one
    cooperative launch (a5g_set_ctas on each member), each group with its own
    barrier; every member still ends bit-identical to the run driven alone on
    one block."""
    cfgs = _members()
    ctas = [1, 3, 2, 4, 1]
    batch = [streamer.Simulation(c) for c in cfgs]
    alone = [streamer.Simulation(c) for c in cfgs]
    for s, m in zip(batch, ctas):
        s.device.set_ctas(m)
    for s in batch + alone:
        s.init()
    nb, gpu_ms, _, cu = streamer.run_batch(batch, [c.end_time for c in cfgs], use_graph=use_graph,
                                           n_threads=4)
    assert nb > 0 and cu > 0
    for k, (s, c) in enumerate(zip(alone, cfgs)):
        s.run(c.end_time)
        _same(batch[k], s, f"member {k} ({ctas[k]} blocks)")
