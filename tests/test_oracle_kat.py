"""Pins of the CPU oracle against the reference's own known-answer cases.

The reference ships no golden numbers; its multigrid and lookup-table
examples print residuals and errors that must behave in a known way:
  * afivo/examples/multigrid/test_mg2_2d.f90 and test_mg_cyl.f90: the
    residual falls by a large factor every FMG cycle and the error settles
    at the discretization error;
  * fosito/test/test_m_lookup_table.f90: second-order convergence of the
    table interpolation;
  * afivo/examples/transport/test_drift_diff_2d.f90: the exact advected
    solution on an adaptive periodic mesh (bounded error, conserved sum on a
    frozen mesh, second-order convergence on uniform meshes), which pins the
    transport half (fluxes, flux consistency, restriction, ghost cells,
    prolongation, refinement);
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


def test_drift_diff_known_answer():
    """afivo/examples/transport/test_drift_diff_2d.f90 (its own parameters:
    velocity (1, 1), no diffusion, trapezoidal steps, a regrid after every
    step, t = 5): the transport half of the oracle -- Koren fluxes with the
    second ghost layer, flux consistency at refinement boundaries,
    restriction, limited ghost cells, prolongation of new boxes -- follows the
    exact advected solution sin^4(x - t) cos^4(y - t)."""
    r = a5ref.kat_drift_diff(0, 5.0, True)
    assert r["time"] > 5.0 and r["steps"] > 800
    assert r["max_lvl"] == 6                 # dr = 2 pi / 256 where the solution varies fastest
    assert r["max_err"] < 0.02               # measured 0.0128
    assert r["mean_err"] < 2.0e-3            # measured 1.4e-3
    # the regrids prolong linearly (not conservatively): the sum drifts slowly
    assert abs(r["sum_end"] - r["sum0"]) / r["sum0"] < 0.01


def test_drift_diff_conserves_on_a_frozen_mesh():
    """Without regrids the finite-volume update with consistent fluxes on the
    periodic square conserves the sum of phi to rounding."""
    r = a5ref.kat_drift_diff(0, 1.0, False)
    assert r["max_lvl"] == 6 and r["steps"] > 150
    assert abs(r["sum_end"] - r["sum0"]) / r["sum0"] < 1e-13


def test_drift_diff_second_order_on_uniform_meshes():
    """Uniform meshes of levels 3, 4, 5 to t = 1: the mean error falls by
    about 4 per level (Koren's scheme is second order away from extrema), and
    the initial sum approaches the integral (3 pi / 4)^2."""
    errs = [a5ref.kat_drift_diff(lvl, 1.0, True) for lvl in (3, 4, 5)]
    for a, b in zip(errs, errs[1:]):
        assert a["mean_err"] / b["mean_err"] > 3.5, (a["mean_err"], b["mean_err"])
        assert a["max_err"] / b["max_err"] > 2.2
    assert abs(errs[-1]["sum0"] - (0.75 * math.pi) ** 2) < 1e-3
    for r in errs:
        assert abs(r["sum_end"] - r["sum0"]) / r["sum0"] < 1e-13


def test_tree_sum_cc_formula():
    """a$D_tree_sum_cc (afivo/src/m_aX_utils.f90:621-680) with one thread:
    the oracle's value equals the plain loop over levels, leaves and cells of
    lvl_dr^2 times the box sum (cylindrical: 2 pi r times the value)."""
    for cfg in (config.cartesian_8mm(), config.cylindrical_16mm()):
        sim = a5ref.Sim(cfg, n_threads=2)
        sim.init()
        meta, geom, levels = sim.meta(), sim.geom(), sim.levels()
        x = sim.cc(a5ref.I_ELEC)
        total = 0.0
        for lvl in sorted(levels):
            leaves = levels[lvl][1]
            dr = cfg.dr_base * 0.5 ** (lvl - 1)
            for id_ in leaves:
                n = int(meta[id_, 14])
                g = n + 2
                tmp = 0.0
                for j in range(1, n + 1):
                    for i in range(1, n + 1):
                        v = float(x[id_, i + g * j])
                        tmp = tmp + (v * (geom[id_, 0] + (i - 0.5) * geom[id_, 3]) if cfg.coord == "cyl" else v)
                if cfg.coord == "cyl":
                    tmp = tmp * (2 * math.acos(-1.0))
                total = total + dr * dr * tmp
        assert sim.tree_sum_cc(a5ref.I_ELEC, 1) == total


def test_mg3_2d_layered_dielectric_known_answer():
    """afivo/examples/multigrid/test_mg3_2d.f90: eps jumps from 1 to 4 at
    y = 0.5 (a cell face on every level). With the harmonic face weights of
    the eps operators the layered solution (1.6 y below, 0.8 + 0.4 (y - 0.5)
    above) satisfies the discrete equations exactly, so the multigrid must
    converge to it to rounding -- across the refinement boundaries of the
    level-7 patch around the centre as well."""
    res, err, max_lvl, n_leaf = a5ref.kat_mg3_2d(8)
    assert max_lvl == 7 and n_leaf > 300
    for k in range(3):
        assert res[k + 1] < res[k] / 10.0
    assert err[0] < 1e-7
    assert max(err[4:]) < 1e-13


def test_mgb_2d_level_set_known_answer():
    """afivo/examples/multigrid/test_mgb_2d.f90: internal boundaries from a
    level set (value 1e3 on the zero contour). For the plane y = 1.3 the
    one-sided differences of the level-set operators are exact for the
    piecewise-linear solution, so the multigrid converges to it to rounding;
    for the example's own ellipse the residual falls by a large factor per
    cycle."""
    res, err, n_lsf = a5ref.kat_mgb_2d("plane", 12)
    assert n_lsf > 30
    for k in range(6):
        assert res[k + 1] < res[k] / 10.0
    assert err[-1] < 1e-12 * 1e3
    res, _, n_lsf = a5ref.kat_mgb_2d("ellipse", 10)
    assert n_lsf > 60
    for k in range(7):
        assert res[k + 1] < res[k] / 10.0
