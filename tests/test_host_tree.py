"""The product's host quadtree (include/a5t.h) against the oracle's tree:
given the same refinement flags it must make the same topology decisions
(refine, 2:1 balance, derefine, neighbour links, level lists, new ids)."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config, streamer
from a5_streamer_b200._lib import lib

CASES = {
    "cart": config.cartesian_8mm(),
    "cyl": config.cylindrical_16mm(),
    "cart_active": config.cartesian_8mm(applied_fld=7e6, lvls_max=6),
}


def _product_tree(cfg):
    t = streamer.Tree(cfg.box_size, cfg.lvls_max, cfg.dr_base, (0.0, 0.0),
                      1 if cfg.coord == "cyl" else 0)
    ix, nb = streamer.base_grid(cfg.n_base)
    t.set_base(ix, nb)
    return t


def _same(t, sim, where):
    # the invariants the checkpoint loader requires hold for every tree the
    # refinement produces
    assert lib().a5t_check(t.h) == 0, where
    meta, geom, levels = t.export()
    assert np.array_equal(meta, sim.meta()), where
    assert np.array_equal(geom, sim.geom()), where
    rl = sim.levels()
    assert sorted(levels) == sorted(rl), where
    for lvl in levels:
        for a, b in zip(levels[lvl], rl[lvl]):
            assert np.array_equal(a, b), (where, lvl)


@pytest.mark.parametrize("name", sorted(CASES))
def test_tree_decisions_match_oracle(name):
    cfg = CASES[name]
    sim = a5ref.Sim(cfg, n_threads=2)
    t = _product_tree(cfg)
    _same(t, sim, "base")
    # initial refinement loop, then main-loop blocks with regrids
    it = 0
    while True:
        it += 1
        sim.set_init_cond()
        sim.op("compute_fld", 1)
        flags = sim.ref_flags()
        old = sim.max_id
        na, nr = t.adjust_refinement(flags)
        ra, rr = sim.regrid()
        assert (na, nr) == (ra, rr)
        _same(t, sim, f"init {it}")
        new = t.new_boxes()
        meta = sim.meta()
        expect = {}
        for i in range(old + 1, sim.max_id + 1):
            if meta[i, 0]:
                expect.setdefault(int(meta[i, 1]), []).append(i)
        assert {k: v for k, v in new.items() if v} == expect
        if na == 0:
            break
    for k in range(4 if name != "cart_active" else 12):
        dt = sim.get_max_dt()
        for _ in range(cfg.num_steps_amr):
            sim.step(dt)
        flags = sim.ref_flags()
        na, nr = t.adjust_refinement(flags)
        ra, rr = sim.regrid()
        assert (na, nr) == (ra, rr)
        if ra or rr:
            sim.op("compute_fld", 0)
        _same(t, sim, f"block {k}")


def test_derefinement_after_seed_window():
    # past the seed-refinement window the seed boxes are coarsened again
    cfg = config.cartesian_8mm()
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    t = _product_tree(cfg)
    # replay the oracle's initial loop on the product tree
    s2 = a5ref.Sim(cfg, n_threads=2)
    while True:
        s2.set_init_cond()
        s2.op("compute_fld", 1)
        na, _ = t.adjust_refinement(s2.ref_flags())
        s2.regrid()
        if na == 0:
            break
    sim.time = 5e-9
    s2.time = 5e-9
    before = s2.max_lvl
    na, nr = t.adjust_refinement(s2.ref_flags())
    s2.regrid()
    assert nr > 0 and na == 0
    assert t.max_lvl == s2.max_lvl <= before
    _same(t, s2, "derefine")


def test_bad_base_rejected():
    from a5_streamer_b200._lib import A5GError
    t = streamer.Tree(8, 5, 1.0, (0.0, 0.0), 0)
    with pytest.raises(A5GError):
        t.set_base(np.array([[0, 1]]), np.array([[-1, -1, -1, -1]]))
