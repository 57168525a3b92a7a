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


@pytest.mark.parametrize("name", ["cartesian_8mm", "cylindrical_16mm", "cylindrical_16mm_photoi"])
def test_run_to_end_time(name):
    """Whole runs from the initial conditions to the end time, regrids
    included. cylindrical_16mm_photoi is the benchmark's workload (the mesh
    bench.py times: levels -1..7 at t = 10 ns) with Monte Carlo
    photoionization, reproduced for the oracle's stated team size."""
    cfg = {"cartesian_8mm": config.cartesian_8mm(),
           "cylindrical_16mm": config.cylindrical_16mm(),
           "cylindrical_16mm_photoi": config.cylindrical_16mm(photoi=True)}[name]
    sim = streamer.Simulation(cfg)
    ref = a5ref.Sim(cfg, n_threads=4)
    sim.init(); ref.init()
    nb1 = sim.run(cfg.end_time)
    nb2 = ref.run(cfg.end_time)
    assert nb1 == nb2
    assert sim.time == ref.time and sim.time > cfg.end_time
    _compare_full(sim, ref, "end")
    if cfg.photoi_enabled:
        meta = ref.meta()
        m = side_mask(meta, cfg.box_size)
        assert np.array_equal(sim.device.cc(7)[m], ref.cc(7)[m]), "photoionization source differs"
        assert np.array_equal(sim.device.rng_state(), ref.rng_state())
    assert sim.device.n_leaf_cells() == ref.n_leaf_cells()
