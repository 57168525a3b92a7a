"""Known answers of the 3D octree form of the oracle (no GPU): the
reference's 3D multigrid and transport examples, restated on uniformly
refined octrees, pin the oracle's 3D box operators, ghost cells,
restriction, FAS cycles, Koren fluxes and trapezoidal step."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config


def test_mg2_3d_residual_falls_each_cycle():
    """afivo/examples/multigrid/test_mg2_3d.f90: each FAS-FMG cycle reduces
    the residual by a large factor until rounding."""
    for level in (3, 4):
        res, err = a5ref.kat_mg3(level, 6)
        for c in range(5):
            assert res[c + 1] < res[c] / 20, (level, c, res)
        # the error settles at the discretisation error
        assert abs(err[-1] - err[-2]) <= 1e-3 * err[-1]


def test_mg2_3d_second_order():
    """The discretisation error of the manufactured two-Gaussian solution
    falls toward second order as the mesh resolves sigma = 0.05 (h = 1/32,
    1/64, 1/128 at levels 3..5)."""
    errs = [a5ref.kat_mg3(level, 4)[1][-1] for level in (3, 4, 5)]
    assert errs[0] > errs[1] > errs[2]
    assert errs[1] / errs[2] > 3.4, errs
    assert errs[2] < 0.01


def test_drift_diff_3d_converges_and_conserves():
    """afivo/examples/transport/test_drift_diff_3d.f90: advection of
    sin^4(x - t) cos^4(z - t) on the periodic cube with Koren fluxes and the
    trapezoidal step; the sum of phi is conserved to rounding and the error
    is second order in the mean."""
    out = [a5ref.kat_drift_diff3(level, 1.0) for level in (2, 3, 4)]
    for r in out:
        assert abs(r["sum_end"] - r["sum0"]) <= 1e-13 * abs(r["sum0"])
        assert r["time"] >= 1.0
    means = [r["mean_err"] for r in out]
    assert means[0] / means[1] > 3.0 and means[1] / means[2] > 3.5, means
    assert out[-1]["max_err"] < 0.06


def test_3d_oracle_runs_the_streamer_step():
    """The 3D streamer on a level-2 uniform octree: the initial loop stops at
    the uniform level, the step keeps the densities finite and conserves
    charge where no source acts (the step only moves electrons)."""
    cfg = config.cube_16mm_uniform(2)
    sim = a5ref.Sim3(cfg, n_threads=2)
    assert sim.init() == 2
    assert (sim.min_lvl, sim.max_lvl, sim.max_id) == (-1, 2, 11)
    dt = sim.get_max_dt()
    assert 0 < dt <= cfg.dt_max / 2
    fld0 = sim.dt_reductions()
    sim.step(dt)
    assert np.all(np.isfinite(sim.cc(0)))
    assert sim.dt_reductions()[0] > 0.9 * fld0[0]
    # the applied potential on the high-z wall
    assert sim.applied_voltage == pytest.approx(-16e-3 * 2e6)


def test_3d_config_rules():
    cfg = config.cube_16mm_uniform(4)
    cfg.validate()
    with pytest.raises(ValueError):
        config.cube_16mm_uniform(4, uniform_lvl=0).validate()
    with pytest.raises(ValueError):
        config.cube_16mm_uniform(4, epsilon_diel=2.0).validate()
    with pytest.raises(ValueError):
        config.cube_16mm_uniform(4, domain_len=(16e-3, 8e-3, 16e-3)).validate()
