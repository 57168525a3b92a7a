"""Pins of the CPU oracle against the reference's own known-answer cases.

The reference ships no golden numbers; its multigrid and lookup-table
examples print residuals and errors that must behave in a known way:
  * afivo/examples/multigrid/test_mg2_2d.f90 and test_mg_cyl.f90: the
    residual falls by a large factor every FMG cycle and the error settles
    at the discretization error;
  * fosito/test/test_m_lookup_table.f90: second-order convergence of the
    table interpolation;
  * src/m_streamer.f90:339-362: the four branches of koren_mlim;
plus a manufactured solution solved with the streamer's own boundary
conditions (grounded bottom, applied voltage on top, Neumann sides) on the
streamer's own tree."""
import math

import numpy as np

import a5ref
from a5_streamer_b200 import config


def test_mg2_2d_known_answer():
    res, err, max_lvl, cells = a5ref.kat_mg(False, 8)
    assert max_lvl >= 8 and cells > 50000
    for k in range(5):
        assert res[k + 1] < res[k] / 10.0
    assert res[-1] < 1e-6
    assert 5e-5 < err[-1] < 2e-4           # settled discretization error
    assert abs(err[-1] - err[-2]) < 1e-9


def test_mg_cyl_known_answer():
    res, err, max_lvl, cells = a5ref.kat_mg(True, 8)
    assert max_lvl == 6
    assert res[3] < 1e-6 and res[-1] < 1e-9
    assert err[-1] < 2e-4


def test_mg_cyl_diel_known_answer():
    """afivo/examples/multigrid/test_mg_cyl_diel.f90: a jump of eps (100 vs 1)
    with surface charge; the eps operators (gsrb_clpld, clpld, corr_lpld)
    converge to the manufactured solution at the discretization error."""
    res, err, max_lvl, n_diel = a5ref.kat_mg_diel(6)
    assert n_diel > 100 and max_lvl >= 8
    for k in range(4):
        assert res[k + 1] < res[k] / 10.0
    assert err[-1] < 2e-4
    assert abs(err[-1] - err[-2]) < 1e-8


def test_lookup_table_second_order():
    errs = [a5ref.kat_lookup(n) for n in (20, 40, 80, 160, 320)]
    ratios = [errs[k + 1] / errs[k] for k in range(len(errs) - 1)]
    for r in ratios:
        assert 0.2 < r < 0.3, ratios


def test_koren_limiter_branches():
    k = a5ref.koren_mlim
    assert k(1.0, -1.0) == 0.0 and k(0.0, 1.0) == 0.0
    assert k(0.1, 1.0) == 0.1                       # a/b <= 1/4: a
    assert k(1.0, 1.0) == (1 / 6.0) * (1.0 + 2 * 1.0)  # 1/4 < a/b <= 2.5
    assert k(3.0, 1.0) == 1.0                       # a/b > 2.5: b


def test_manufactured_poisson_streamer_bcs():
    cfg = config.cartesian_8mm()
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    L = cfg.domain_len_z
    V = cfg.applied_voltage
    A = 1.0e3
    meta, geom = sim.meta(), sim.geom()
    nc = cfg.box_size
    rhs = np.zeros((meta.shape[0], (nc + 2) ** 2))
    exact = np.zeros_like(rhs)
    mask = np.zeros_like(rhs, dtype=bool)
    for i_d in range(1, meta.shape[0]):
        if not meta[i_d, 0]:
            continue
        n = meta[i_d, 14]
        g = n + 2
        dr = geom[i_d, 3]
        x = geom[i_d, 0] + (np.arange(g) - 0.5) * dr
        y = geom[i_d, 1] + (np.arange(g) - 0.5) * dr
        X, Y = np.meshgrid(x, y)  # [j, i]
        phi = V * Y / L + A * np.cos(np.pi * X / L) * np.sin(np.pi * Y / L)
        lap = -2 * (np.pi / L) ** 2 * A * np.cos(np.pi * X / L) * np.sin(np.pi * Y / L)
        rhs[i_d, :g * g] = lap.reshape(-1)
        exact[i_d, :g * g] = phi.reshape(-1)
        m = np.zeros((g, g), dtype=bool)
        m[1:n + 1, 1:n + 1] = True
        if meta[i_d, 1] >= 1:
            mask[i_d, :g * g] = m.reshape(-1)
    sim.set_cc(a5ref.I_RHS, rhs)
    sim.set_cc(a5ref.I_PHI, np.zeros_like(rhs))
    errs = []
    for it in range(6):
        sim.op("fmg", 1, 1 if it == 0 else 0)
        errs.append(np.max(np.abs(sim.cc(a5ref.I_PHI)[mask] - exact[mask])))
    # converged to the discretization error, far below the potential scale
    assert errs[-1] < 1e-3 * abs(V)
    assert abs(errs[-1] - errs[-2]) < 1e-6 * abs(V)
