"""Level-set boundaries of the field solve (a5g_set_level_set; the Afivo
operators mg$D_box_gsrb_lpllsf / _lpllsf / _corr_lpllsf on the boxes the
zero contour crosses) on the device against the oracle, to the bit: a
circular electrode at a fixed potential inside the 8 mm Cartesian domain,
first and later FMG cycles, then whole time steps with it."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config
from parity import compare, device_from_oracle

pytestmark = pytest.mark.gpu


def _electrode(sim, center=(4e-3, 3e-3), radius=0.7e-3, value=-1.5e4):
    meta, geom = sim.meta(), sim.geom()
    nc = sim.nc
    S = (nc + 2) ** 2
    lsf = np.zeros((meta.shape[0], S))
    bval = np.full((meta.shape[0], S), value)
    for b in range(1, meta.shape[0]):
        if not meta[b, 0]:
            continue
        n = int(meta[b, 14])
        g = n + 2
        x = geom[b, 0] + (np.arange(g) - 0.5) * geom[b, 3]
        y = geom[b, 1] + (np.arange(g) - 0.5) * geom[b, 3]
        X, Y = np.meshgrid(x, y)
        lsf[b, :g * g] = (np.sqrt((X - center[0]) ** 2 + (Y - center[1]) ** 2) - radius).reshape(-1)
    return lsf, bval


def _setup():
    cfg = config.cartesian_8mm()
    sim = a5ref.Sim(cfg, n_threads=4)
    sim.init()
    sim.advance(True)
    lsf, bval = _electrode(sim)
    run = device_from_oracle(sim, cfg)
    sim.set_level_set(lsf, bval)
    run.set_level_set(lsf, bval)
    return cfg, sim, run


def test_level_set_fmg_parity():
    cfg, sim, run = _setup()
    sim.op("set_rhs")
    run.set_cc(6, sim.cc(6))
    for first in (1, 0, 0):
        sim.op("fmg", 1, first)
        run.fas_fmg(True, bool(first))
        compare(sim, run, cc_vars=[4, 6], where=f"level-set FMG first={first}")
    phi = sim.cc(4)
    # the electrode holds the potential: cells well inside it are near it
    assert np.min(phi) < -1.0e4


def test_level_set_steps_parity():
    cfg, sim, run = _setup()
    for k in range(2):
        dt = sim.get_max_dt()
        assert run.get_max_dt() == dt
        sim.step(dt)
        run.step(dt)
        compare(sim, run, where=f"level-set step {k}")
