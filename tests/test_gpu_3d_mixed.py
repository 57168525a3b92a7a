"""The mixed-precision form of the 3D octree path (a5g3_set_precision): FP32
fluxes, lookups and multigrid smoothing inside an FP64 defect correction,
against the FP64 path (bit-identical to the oracle) on the same states. The
bounds are the ones the mixed form is held to: max |E| within 1e-4 relative
and the head position within 0.5 % of the FP64 run."""
import numpy as np
import pytest

from a5_streamer_b200 import config, device3

pytestmark = pytest.mark.gpu

N_CC, N_FC = 9, 2


def _copy_state(src, dst):
    for iv in range(N_CC):
        dst.set_cc(iv, src.cc(iv))
    for d in range(3):
        for f in range(N_FC):
            dst.set_fc(d, f, src.fc(d, f))


def _head(run):
    """(max |E|, z of the cell holding it) over the leaves."""
    E = run.cc(5)
    meta = run.meta()
    lvl = run.max_lvl
    g = run.nc + 2
    ids = run.levels()[lvl][0]
    sub = E[ids].reshape(len(ids), g, g, g)[:, 1:-1, 1:-1, 1:-1]
    q = np.unravel_index(np.argmax(sub), sub.shape)
    id_ = ids[q[0]]
    dr = run.cfg.dr_at(lvl)
    z0 = (meta[id_, 4] - 1) * run.nc * dr
    return float(sub[q]), z0 + (q[1] + 0.5) * dr  # sub is [k, j, i] of the slot layout


def _pair(level):
    cfg = config.cube_16mm_uniform(level)
    a = device3.Run3(cfg)
    a.init()
    b = device3.Run3(cfg)
    _copy_state(a, b)
    return cfg, a, b


def test_mixed_field_solve_tracks_fp64():
    cfg, a, b = _pair(4)
    dt = a.get_max_dt()
    for _ in range(4):
        a.step(dt)
    a.sync()
    _copy_state(a, b)
    b.set_precision(True)
    a.compute_fld(False)
    b.compute_fld(False)
    Ea, Eb = a.cc(5), b.cc(5)
    ids = a.levels()[a.max_lvl][0]
    assert np.max(np.abs(Ea[ids] - Eb[ids])) <= 1e-6 * np.max(np.abs(Ea[ids]))
    pa, pb = a.cc(4)[ids], b.cc(4)[ids]
    assert np.max(np.abs(pa - pb)) <= 1e-7 * np.max(np.abs(pa))


@pytest.mark.parametrize("schedule", [None, (0, 1, 1, 4, 2)])
def test_mixed_steps_within_bounds(schedule):
    cfg, a, b = _pair(4)
    b.set_precision(True, schedule)
    for _ in range(10):
        dt = a.get_max_dt()
        for _ in range(cfg.num_steps_amr):
            a.step(dt)
            b.step(dt)
    a.sync()
    b.sync()
    Ea, za = _head(a)
    Eb, zb = _head(b)
    assert np.isfinite(Eb)
    assert abs(Eb - Ea) <= 1e-4 * Ea
    assert abs(zb - za) <= 5e-3 * za
    ne_a, ne_b = a.tree_max_cc(0), b.tree_max_cc(0)
    assert abs(ne_b - ne_a) <= 1e-4 * ne_a


def test_mixed_is_deterministic_and_switchable():
    cfg, a, b = _pair(3)
    c = device3.Run3(cfg)
    _copy_state(a, c)
    for r in (b, c):
        r.set_precision(True)
    dt = a.get_max_dt()
    for _ in range(4):
        b.step(dt)
        c.step(dt)
    b.sync()
    c.sync()
    for iv in (0, 1, 4, 5):
        assert np.array_equal(b.cc(iv), c.cc(iv))
    # back to FP64: the same graph-replayed step as a run that never left it
    b.set_precision(False)
    _copy_state(a, b)
    for _ in range(2):
        a.step(dt)
        b.step(dt)
    a.sync()
    b.sync()
    for iv in (0, 1, 4, 5):
        assert np.array_equal(a.cc(iv), b.cc(iv))
