"""The 3D octree form on the device (include/a5g3.h) against the oracle's
restatement of src/streamer_3d.f90 and afivo's m_a3_* routines, on a
uniformly refined octree: the same tree (ids, levels, neighbours), then each
operation of the time step from the same state, then whole steps, bit for
bit (tolerance 0: both compute every expression in the reference's order
with separately rounded multiplies and adds)."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config, device3

pytestmark = pytest.mark.gpu

N_CC, N_FC = 9, 2
NAMES = ["n_e", "n_i", "n_e_old", "n_i_old", "phi", "|E|", "rhs", "pho", "eps"]


def _pair(level=3, **kw):
    cfg = config.cube_16mm_uniform(level, **kw)
    sim = a5ref.Sim3(cfg, n_threads=4)
    sim.init()
    rc, xmin, inv, n = sim.table()
    run = device3.Run3(cfg, table=(rc, xmin, inv, n))
    _upload(sim, run)
    return cfg, sim, run


def _upload(sim, run):
    for iv in range(N_CC):
        run.set_cc(iv, sim.cc(iv))
    for d in range(3):
        for f in range(N_FC):
            run.set_fc(d, f, sim.fc(d, f))


def _compare(sim, run, where, ivs=range(N_CC), faces=True):
    for iv in ivs:
        a, b = sim.cc(iv), run.cc(iv)
        bad = np.argwhere(~((a == b) | (np.isnan(a) & np.isnan(b))))
        assert bad.size == 0, (f"{where}: {NAMES[iv]} differs at {len(bad)} entries, first "
                               f"id {bad[0][0]} cell {bad[0][1]}: {a[tuple(bad[0])]!r} vs {b[tuple(bad[0])]!r}")
    if faces:
        for d in range(3):
            for f in range(N_FC):
                a, b = sim.fc(d, f), run.fc(d, f)
                assert np.array_equal(a, b), f"{where}: face {d}/{f} differs ({np.count_nonzero(a != b)} entries)"


def test_tree_matches_reference_construction():
    cfg, sim, run = _pair(3)
    assert (run.max_id, run.min_lvl, run.max_lvl) == (sim.max_id, sim.min_lvl, sim.max_lvl)
    assert np.array_equal(run.meta(), sim.meta())
    lv_s, lv_r = sim.levels(), run.levels()
    assert sorted(lv_s) == sorted(lv_r)
    for lvl in lv_s:
        for a, b in zip(lv_s[lvl], lv_r[lvl]):
            assert np.array_equal(a, b), lvl
    assert run.n_leaf_cells == sim.n_leaf_cells() == 32768


def test_transport_table_matches_oracle():
    cfg = config.cube_16mm_uniform(2)
    sim = a5ref.Sim3(cfg)
    rc, xmin, inv, n = sim.table()
    rc2, xmin2, inv2, n2 = device3.transport_table(cfg)
    assert (n, xmin, inv) == (n2, xmin2, inv2)
    assert np.array_equal(rc, rc2)


@pytest.mark.parametrize("op", ["copy", "fluxes", "update", "restrict", "gc", "average", "set_rhs",
                                "fld_from_pot", "fmg_first", "fmg", "fmg_residual", "vcycle",
                                "compute_fld"])
def test_op_parity(op):
    cfg, sim, run = _pair(3)
    dt = sim.get_max_dt()
    if op == "copy":
        sim.op("copy_cc", 0, 2); run.op("tree_copy_cc", 0, 2)
    elif op == "fluxes":
        sim.op("fluxes_koren", dt); run.op("fluxes_koren", dt)
    elif op == "update":
        sim.op("fluxes_koren", dt); run.op("fluxes_koren", dt)
        sim.op("update_solution", dt); run.op("update_solution", dt)
    elif op == "restrict":
        sim.op("restrict_tree", 0); run.op("restrict_tree", 0)
    elif op == "gc":
        sim.op("gc_tree", 1); run.op("gc_tree", 1)
    elif op == "average":
        sim.op("average_dens"); run.op("average_dens")
    elif op == "set_rhs":
        sim.op("set_rhs"); run.op("set_rhs")
    elif op == "fld_from_pot":
        sim.op("fld_from_pot"); run.op("fld_from_pot")
    elif op == "fmg_first":
        sim.op("set_rhs"); run.op("set_rhs")
        sim.op("fmg", 0, 1); run.op("fmg", 0, 1)
    elif op == "fmg":
        sim.op("set_rhs"); run.op("set_rhs")
        sim.op("fmg", 0, 0); run.op("fmg", 0, 0)
    elif op == "fmg_residual":
        sim.op("set_rhs"); run.op("set_rhs")
        sim.op("fmg", 1, 0); run.op("fmg", 1, 0)
    elif op == "vcycle":
        sim.op("set_rhs"); run.op("set_rhs")
        sim.op("vcycle", sim.max_lvl, 1); run.op("vcycle", run.max_lvl, 1)
    elif op == "compute_fld":
        sim.op("compute_fld", 0); run.compute_fld(False)
    run.sync()
    _compare(sim, run, op)


def test_reductions_and_dt():
    cfg, sim, run = _pair(3)
    assert np.array_equal(run.dt_reductions(), sim.dt_reductions())
    assert run.get_max_dt() == sim.get_max_dt()
    for iv in (0, 5, 6):
        assert run.tree_max_cc(iv) == sim.tree_max_cc(iv)
        assert run.tree_min_cc(iv) == sim.tree_min_cc(iv)


@pytest.mark.parametrize("level", [2, 3])
def test_steps_parity(level):
    """Whole steps (the graph-replayed a5g3_step) from the oracle's initial
    state, dt from get_max_dt each block, as the main loop advances."""
    cfg, sim, run = _pair(level)
    for _ in range(3):
        dt = sim.get_max_dt()
        assert run.get_max_dt() == dt
        for _ in range(cfg.num_steps_amr):
            sim.step(dt)
            run.step(dt)
    run.sync()
    _compare(sim, run, f"after 6 steps (level {level})")


def test_device_init_close_to_reference():
    """The device's own initial conditions (CUDA exp in the seed shape) and
    first field solve agree with the oracle's to rounding."""
    cfg = config.cube_16mm_uniform(3)
    sim = a5ref.Sim3(cfg, n_threads=4)
    sim.init()
    run = device3.Run3(cfg)
    run.init()
    run.sync()
    for iv in (0, 4, 5):
        a, b = sim.cc(iv), run.cc(iv)
        scale = np.max(np.abs(a))
        assert np.max(np.abs(a - b)) <= 1e-12 * scale, NAMES[iv]


def test_rejects_bad_parameters():
    from a5_streamer_b200 import _lib
    p = device3.make_params3(config.cube_16mm_uniform(2))
    p.box_size = 16
    import ctypes
    h = ctypes.c_void_p()
    assert _lib.lib().a5g3_create(ctypes.byref(p), ctypes.byref(h)) == _lib.A5G_EINVAL
    assert b"box_size" in _lib.lib().a5g3_last_error()
