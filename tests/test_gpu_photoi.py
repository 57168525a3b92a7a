"""Monte Carlo photoionization on the device against the oracle, bit for bit:
the photon source term of one call (with and without dt, several team
sizes), the master generator state, whole time steps with photoionization,
the batched step, and whole driver runs with regrids."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config, device as dv, streamer
from parity import compare, device_from_oracle, side_mask

pytestmark = pytest.mark.gpu


def _setup(team, **kw):
    cfg = config.cylindrical_16mm(photoi=True, photoi_team=team, **kw)
    ref = a5ref.Sim(cfg, n_threads=4)
    ref.init()
    run = device_from_oracle(ref, cfg)
    dist, frac, _ = ref.photon_table()
    run.set_photon_table(dist, frac)
    run.set_rng_state(ref.rng_state())
    return cfg, ref, run


def _check_pho(ref, run, where):
    meta = ref.meta()
    m = side_mask(meta, ref.nc)
    a, b = ref.cc(a5ref.I_PHO), run.cc(dv.I_PHO)
    assert np.array_equal(a[m], b[m]), f"{where}: photoionization source differs " \
        f"({int((a[m] != b[m]).sum())} cells)"
    assert np.array_equal(ref.rng_state(), run.rng_state()), f"{where}: generator state differs"


@pytest.mark.parametrize("team", [1, 37, 512, 1000, 148 * 256])
@pytest.mark.parametrize("with_dt", [False, True])
def test_photoionization_call(team, with_dt):
    cfg, ref, run = _setup(team)
    dt = ref.get_max_dt() if with_dt else None
    ref.photoionization(dt)
    run.photoionization(dt)
    run.sync()
    _check_pho(ref, run, f"team {team}")
    assert float(np.abs(ref.cc(a5ref.I_PHO)).sum()) > 0


def test_photoionization_repeated_calls():
    cfg, ref, run = _setup(300)
    for k in range(4):
        dt = 1e-12 * (k + 1)
        ref.photoionization(dt)
        run.photoionization(dt)
        _check_pho(ref, run, f"call {k}")


def test_photoionization_unclean_seed():
    """A caller-set seed outside the generator's invariant range [0, m) is
    stepped draw by draw until it enters it."""
    cfg, ref, run = _setup(64)
    seed = np.array([-2000000000, 2147483600, 5, -7], dtype=np.int32)
    ref.set_rng_state(seed)
    run.set_rng_state(seed)
    ref.photoionization(2e-12)
    run.photoionization(2e-12)
    _check_pho(ref, run, "unclean seed")


def test_step_with_photoionization():
    cfg, ref, run = _setup(148 * 256)
    for k in range(3):
        dt = ref.get_max_dt()
        assert run.get_max_dt() == dt
        ref.step(dt)
        run.step(dt)
        compare(ref, run, where=f"step {k}")
        _check_pho(ref, run, f"step {k}")


def test_photoionization_unreduced_seed():
    """A seed whose lag state lies outside [0, m): the first draws are stepped
    one by one until the state is reduced, before any precomputed jump."""
    cfg, ref, run = _setup(512)
    dirty = (-5, 2147483600, 7, 11)
    ref.set_rng_state(dirty)
    run.set_rng_state(dirty)
    for k in range(2):
        dt = ref.get_max_dt()
        ref.step(dt)
        run.step(dt)
        compare(ref, run, where=f"step {k}")
        _check_pho(ref, run, f"step {k}")


def test_step_batch_with_photoionization():
    cfgs = [config.cylindrical_16mm(photoi=True, photoi_team=t, rng_seed=s)
            for t, s in ((512, (521288629, 362436069, 16163801, 1131199299)),
                         (2000, (1, 2, 3, 4)))]
    cfgs.append(config.cylindrical_16mm())
    refs, runs = [], []
    for cfg in cfgs:
        ref = a5ref.Sim(cfg, n_threads=4)
        ref.init()
        run = device_from_oracle(ref, cfg)
        if cfg.photoi_enabled:
            dist, frac, _ = ref.photon_table()
            run.set_photon_table(dist, frac)
            run.set_rng_state(ref.rng_state())
        refs.append(ref)
        runs.append(run)
    for k in range(2):
        dts = [r.get_max_dt() for r in refs]
        for r, dt in zip(refs, dts):
            r.step(dt)
        dv.step_batch(runs, dts)
        for r, d in zip(refs, runs):
            d.sync()
            compare(r, d, where=f"batch step {k}")
            if r.cfg.photoi_enabled:
                _check_pho(r, d, f"batch step {k}")


def test_driver_run_with_photoionization():
    cfg = config.cylindrical_16mm(photoi=True)
    sim = streamer.Simulation(cfg)
    ref = a5ref.Sim(cfg, n_threads=4)
    assert sim.init() == ref.init()
    for k in range(3):
        dt1 = sim.advance(True)
        dt2 = ref.advance(True)
        assert dt1 == dt2, (k, dt1, dt2)
        meta, geom, _ = sim.tree.export()
        assert np.array_equal(meta, ref.meta())
        m = side_mask(meta, cfg.box_size)
        for iv in (0, 1, 4, 7):
            a, b = sim.device.cc(iv), ref.cc(iv)
            assert np.array_equal(a[m], b[m]), f"block {k}: variable {iv} differs"
