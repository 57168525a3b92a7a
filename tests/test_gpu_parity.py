"""Device path vs CPU oracle, operation by operation and step by step, on the
8 mm Cartesian case and the cylindrical case (seeded, deterministic inputs).
Integer results must match exactly; floating-point state must match to the
bit (both sides round every operation separately: no FMA contraction)."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config
from a5_streamer_b200 import device as dv
from parity import compare, device_from_oracle

pytestmark = pytest.mark.gpu


def _cases():
    return {
        "cart": config.cartesian_8mm(),
        "cyl": config.cylindrical_16mm(),
    }


@pytest.fixture(params=["cart", "cyl"], scope="module")
def case(request):
    cfg = _cases()[request.param]
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    for _ in range(2):
        sim.advance(True)
    return cfg, sim


def _fresh(case):
    cfg, sim0 = case
    # independent copy of the oracle state: replay the same deterministic run
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    for _ in range(2):
        sim.advance(True)
    run = device_from_oracle(sim, cfg)
    compare(sim, run, where="upload")
    return cfg, sim, run


DT = 2.5e-11


@pytest.mark.parametrize("op", ["copy", "fluxes", "consistent", "update", "restrict",
                                "gc_lim", "gc_interp", "average", "fld_from_pot",
                                "fmg_first", "compute_fld"])
def test_op_parity(case, op):
    cfg, sim, run = _fresh(case)
    if op == "copy":
        sim.op("copy_cc", 0, 2); run.tree_copy_cc(0, 2)
    elif op == "fluxes":
        sim.op("fluxes_koren", DT); run.fluxes_koren(DT)
    elif op == "consistent":
        sim.op("fluxes_koren", DT); run.fluxes_koren(DT)
        sim.op("consistent_fluxes"); run.consistent_fluxes()
    elif op == "update":
        sim.op("fluxes_koren", DT); run.fluxes_koren(DT)
        sim.op("consistent_fluxes"); run.consistent_fluxes()
        sim.op("update_solution", DT); run.update_solution(DT)
    elif op == "restrict":
        sim.op("restrict_tree", 0); run.restrict_tree(0)
    elif op == "gc_lim":
        sim.op("restrict_tree", 1); run.restrict_tree(1)
        sim.op("gc_tree", 1, 0); run.gc_tree(1, 0)
    elif op == "gc_interp":
        sim.op("gc_tree", 5, 1); run.gc_tree(5, 1)
    elif op == "average":
        sim.op("average_dens"); run.average_dens()
    elif op == "fld_from_pot":
        sim.op("fld_from_pot"); run.fld_from_pot()
    elif op == "fmg_first":
        sim.op("fmg", 0, 1); run.fas_fmg(False, True)
        # tmp (the |E| variable) is multigrid scratch: on parent boxes it
        # holds the applied correction in the reference, not here
        compare(sim, run, cc_vars=[0, 1, 2, 3, 4, 6, 7, 8], where=op)
        return
    elif op == "compute_fld":
        sim.op("compute_fld", 0); run.compute_fld(False)
    compare(sim, run, where=op)


def test_fmg_after_rhs(case):
    cfg, sim, run = _fresh(case)
    sim.op("set_rhs")
    run.set_cc(6, sim.cc(6))
    sim.op("fmg", 0, 0)
    run.fas_fmg(False, False)
    compare(sim, run, cc_vars=[4, 6], where="fmg")


def test_fmg_set_residual(case):
    cfg, sim, run = _fresh(case)
    sim.op("set_rhs")
    run.set_cc(6, sim.cc(6))
    sim.op("fmg", 1, 0)
    run.fas_fmg(True, False)
    # with set_residual the residual of every box is left in tmp
    compare(sim, run, cc_vars=[4, 6], where="fmg_res")
    from parity import interior_mask
    m = interior_mask(sim.meta(), cfg.box_size)
    assert np.array_equal(sim.cc(5)[m], run.cc(5)[m])


@pytest.mark.parametrize("below_top", [0, 2])
@pytest.mark.parametrize("set_residual", [False, True])
def test_vcycle_parity(case, below_top, set_residual):
    """mg$D_fas_vcycle alone (a5g_mg_fas_vcycle): from the state after a
    field solve (valid potential ghost cells, as the routine requires), one
    V-cycle from the finest level or from two levels below it."""
    cfg, sim, run = _fresh(case)
    sim.op("compute_fld", 0)
    run.compute_fld(False)
    max_lvl = sim.max_lvl - below_top
    for k in range(2):
        sim.op("vcycle", max_lvl, int(set_residual))
        run.fas_vcycle(max_lvl, set_residual)
        compare(sim, run, cc_vars=[0, 1, 4, 6], where=f"vcycle {k}")
    if set_residual:
        # the residual of levels min..max_lvl is left in tmp (|E| elsewhere)
        from parity import interior_mask
        m = interior_mask(sim.meta(), cfg.box_size)
        assert np.array_equal(sim.cc(5)[m], run.cc(5)[m])


@pytest.mark.parametrize("iv", [0, 1, 4, 5])
def test_tree_reductions(case, iv):
    """a$D_tree_max_cc / _min_cc / _sum_cc over the leaves; the sum as teams
    of several sizes form it."""
    cfg, sim, run = _fresh(case)
    assert run.tree_max_cc(iv) == sim.tree_max_cc(iv)
    assert run.tree_min_cc(iv) == sim.tree_min_cc(iv)
    for team in (1, 3, 64, 1000):
        assert run.tree_sum_cc(iv, team) == sim.tree_sum_cc(iv, team), team


def test_dt_and_flags(case):
    cfg, sim, run = _fresh(case)
    assert np.array_equal(sim.dt_reductions(), run.dt_reductions())
    assert sim.get_max_dt() == run.get_max_dt()
    for t in (0.0, 10e-9):
        sim.time = t
        f_o = sim.ref_flags()
        f_d = run.ref_flags(t)
        assert np.array_equal(f_o, f_d), np.flatnonzero(f_o != f_d)


def test_step_parity(case):
    cfg, sim, run = _fresh(case)
    for k in range(3):
        dt = sim.get_max_dt()
        assert dt == run.get_max_dt()
        sim.step(dt)
        run.step(dt)
        compare(sim, run, where=f"step {k}")


def test_regrid_prolong_parity(case):
    cfg, sim, run = _fresh(case)
    old_max = sim.max_id
    sim.time = 0.0
    n_add, n_rm = sim.regrid()
    meta = sim.meta()
    run.upload_tree(meta, sim.geom(), sim.min_lvl, sim.max_lvl, sim.levels())
    new = {}
    for id_ in range(old_max + 1, sim.max_id + 1):
        if meta[id_, 0]:
            new.setdefault(int(meta[id_, 1]), []).append(id_)
    run.prolong_to_new_boxes(new)
    compare(sim, run, cc_vars=[0, 1, 4, 8], fc_vars=(), where="prolong")


def test_batch_matches_single(case):
    cfg, sim, run = _fresh(case)
    run_b = device_from_oracle(sim, cfg)
    run_c = device_from_oracle(sim, cfg)
    dt = sim.get_max_dt()
    run.step(dt)
    dv.step_batch([run_b, run_c], [dt, dt])
    run_b.sync()
    for iv in range(9):
        a, b, c = run.cc(iv), run_b.cc(iv), run_c.cc(iv)
        assert np.array_equal(a, b) and np.array_equal(a, c)
