"""The device path's plans and phase schedule, checked on the CPU.

The plans (cell tables with neighbour codes, ghost recipes, restriction and
residual-restriction records) come from the library's host-only builder; the
multigrid phases are replayed by tests/plan_emulator.py exactly as the device
runs them (all outputs of a phase from the state before it, same arithmetic
order). The result must equal the oracle's FAS FMG bit for bit, on trees that
include refinement boundaries, physical corners, removed boxes and a full
finest level (lvls_max reached)."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config
from parity import interior_mask, side_mask
from plan_emulator import Emulator, Plans

CASES = {
    "cart": (config.cartesian_8mm(), 2),
    "cyl": (config.cylindrical_16mm(), 2),
    "cart_active_1": (config.cartesian_8mm(applied_fld=7e6, lvls_max=6), 1),
    "cart_active_2": (config.cartesian_8mm(applied_fld=7e6, lvls_max=6), 2),
    "cart_active_6": (config.cartesian_8mm(applied_fld=7e6, lvls_max=6), 6),
}


def _setup(name):
    cfg, blocks = CASES[name]
    sim = a5ref.Sim(cfg, n_threads=4)
    sim.init()
    for _ in range(blocks):
        sim.advance(True)
    meta, geom, levels = sim.meta(), sim.geom(), sim.levels()
    coord = 1 if cfg.coord == "cyl" else 0
    P = Plans(meta, geom, levels, sim.min_lvl, sim.max_lvl, cfg.dr_base)
    em = Emulator(P, [sim.cc(i) for i in range(9)], coord, cfg.applied_voltage, cfg.n_cycle_base)
    return cfg, sim, meta, em


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("first_call", [False, True])
def test_emulated_fmg_matches_oracle(name, first_call):
    cfg, sim, meta, em = _setup(name)
    sim.op("set_rhs")
    sim.op("fmg", 0, 1 if first_call else 0)
    em.fmg(first_call, True)
    m = side_mask(meta, cfg.box_size).reshape(-1)
    mi = interior_mask(meta, cfg.box_size).reshape(-1)
    assert np.array_equal(sim.cc(4).reshape(-1)[m], em.cc[4][m])
    assert np.array_equal(sim.cc(6).reshape(-1)[mi], em.cc[6][mi])


def test_plan_sizes():
    cfg, sim, meta, em = _setup("cart_active_2")
    P = em.P
    used = [i for i in range(1, meta.shape[0]) if meta[i, 0]]
    assert P.bx_off[P.nlev] == len(used)
    assert sorted(P.boxes["base"][:len(used)] // 100) == sorted(used)
    n_par = sum(len(c) for (_, _, c) in sim.levels().values())
    assert P.pb_off[P.nlev] == n_par
    # the finest level of this tree is lvls_max: its boxes are not listed as
    # leaves (a reference quirk kept for parity)
    top = P.boxes[P.bx_off[P.nlev - 1]:P.bx_off[P.nlev]]
    assert sim.max_lvl == cfg.lvls_max and not (top["flags"] & 1).any()


@pytest.mark.parametrize("name", sorted(CASES))
def test_flat_fill_equals_level_by_level_fill(name):
    """After the oracle's FMG every level's ghost cells hold the level-by-level
    fill of the final potential. The one-phase fill of the mixed form's
    accumulation (phi_ghost_flat: the refinement-boundary source read from
    the parent's same-level neighbour) must give exactly those values, from
    the interior cells alone."""
    cfg, sim, meta, em = _setup(name)
    sim.op("set_rhs")
    sim.op("fmg", 0, 0)
    phi = np.array(sim.cc(4), dtype=np.float64).reshape(-1)
    n_rb = 0
    for lvl in range(em.P.min_lvl, em.P.max_lvl + 1):
        li, nc, ncg, boxes, dr = em.lvl(lvl)
        if len(boxes) == 0:
            continue
        B, side, k = em.ghosts(boxes, nc)
        d = em.ghost_dst(B, nc, ncg, side, k)
        v = em.phi_ghost_flat(phi, B, nc, ncg, side, k)
        assert np.array_equal(v, phi[d]), lvl
        n_rb += int((B["nb"][np.arange(len(B)), side] == -1).sum())
    # the trees have refinement boundaries, so the flat source is exercised
    assert n_rb > 0
