"""The product's own driver (host tree + device data) against the oracle over
whole runs with regrids: identical trees (integer topology and refinement
decisions, to the bit), identical step sizes and identical states."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config, streamer
from parity import interior_mask, side_mask

pytestmark = pytest.mark.gpu

CASES = {
    "cart": (config.cartesian_8mm(), 4),
    "cyl": (config.cylindrical_16mm(), 4),
    # stronger field: the streamer grows, boxes are refined and removed
    "cart_active": (config.cartesian_8mm(applied_fld=7e6, lvls_max=6), 16),
}


def _compare_full(sim, ref, where):
    meta, geom, levels = sim.tree.export()
    assert np.array_equal(meta, ref.meta()), f"{where}: topology differs"
    assert np.array_equal(geom, ref.geom()), f"{where}: geometry differs"
    rl = ref.levels()
    for lvl, (a, b, c) in levels.items():
        ra, rb, rc = rl[lvl]
        assert np.array_equal(a, ra) and np.array_equal(b, rb) and np.array_equal(c, rc), \
            f"{where}: level lists differ at level {lvl}"
    m = side_mask(meta, sim.cfg.box_size)
    mi = interior_mask(meta, sim.cfg.box_size)
    for iv in (0, 1, 2, 3, 4, 8):
        a, b = sim.device.cc(iv), ref.cc(iv)
        assert np.array_equal(a[m], b[m]), f"{where}: variable {iv} differs"
    # |E| interior and side ghosts are rewritten every solve; rhs interior
    assert np.array_equal(sim.device.cc(5)[m], ref.cc(5)[m]), f"{where}: |E| differs"
    assert np.array_equal(sim.device.cc(6)[mi], ref.cc(6)[mi]), f"{where}: rhs differs"


@pytest.mark.parametrize("name", sorted(CASES))
def test_driver_matches_oracle(name):
    cfg, blocks = CASES[name]
    sim = streamer.Simulation(cfg)
    ref = a5ref.Sim(cfg, n_threads=4)
    assert sim.init() == ref.init()
    _compare_full(sim, ref, "init")
    for k in range(blocks):
        dt1 = sim.advance(True)
        dt2 = ref.advance(True)
        assert dt1 == dt2, (k, dt1, dt2)
        assert sim.time == ref.time
        _compare_full(sim, ref, f"block {k}")


def test_run_to_end_time():
    cfg = config.cartesian_8mm()
    sim = streamer.Simulation(cfg)
    ref = a5ref.Sim(cfg, n_threads=4)
    sim.init(); ref.init()
    nb1 = sim.run(cfg.end_time)
    nb2 = ref.run(cfg.end_time)
    assert nb1 == nb2
    _compare_full(sim, ref, "end")
