"""Grid mode (a5g_set_ctas): one run's phases spread over several co-resident
thread blocks of one cooperative launch, with a grid barrier between phases.
The partition of a phase's items over threads changes, the arithmetic does
not: every result must equal the oracle's (and the one-block path's) to the
bit. Also the bounded barrier wait: with a budget of 0 cycles every wait runs
out, the launch returns early and the next synchronising call reports
A5G_TIMEOUT, after which the context works again."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import _lib, config, streamer
from a5_streamer_b200 import device as dv
from parity import compare, device_from_oracle, side_mask

pytestmark = pytest.mark.gpu


def _oracle(cfg, blocks=2):
    sim = a5ref.Sim(cfg, n_threads=4)
    sim.init()
    for _ in range(blocks):
        sim.advance(True)
    return sim


@pytest.mark.parametrize("n_cta,local", [(2, 8192), (7, 0), (148, 8192), (148, 0), (148, 1 << 30)])
@pytest.mark.parametrize("name", ["cart", "cyl"])
def test_grid_step_parity(name, n_cta, local):
    """local: cells up to which a level's phases run on one block of the
    group (0: every phase over all blocks; huge: all levels on one block)."""
    cfg = config.cartesian_8mm() if name == "cart" else config.cylindrical_16mm()
    sim = _oracle(cfg)
    run = device_from_oracle(sim, cfg)
    run.set_ctas(min(n_cta, run.ctas()[1]))
    run.set_grid_local(local)
    for k in range(2):
        dt = sim.get_max_dt()
        assert run.get_max_dt() == dt
        sim.step(dt)
        run.step(dt)
        compare(sim, run, where=f"grid step {k}")
    f_o = sim.ref_flags()
    assert np.array_equal(f_o, run.ref_flags(sim.time))


@pytest.mark.parametrize("op", ["compute_fld", "fmg_first", "vcycle", "gc", "restrict", "fld_from_pot"])
def test_grid_ops(op):
    cfg = config.cylindrical_16mm()
    sim = _oracle(cfg)
    run = device_from_oracle(sim, cfg)
    run.set_ctas(16)
    if op == "compute_fld":
        sim.op("compute_fld", 0); run.compute_fld(False)
    elif op == "fmg_first":
        sim.op("fmg", 0, 1); run.fas_fmg(False, True)
        compare(sim, run, cc_vars=[0, 1, 2, 3, 4, 6, 7, 8], where=op)
        return
    elif op == "vcycle":
        sim.op("vcycle", sim.max_lvl, 1); run.fas_vcycle(sim.max_lvl, True)
        # tmp (the |E| variable) holds the residual on interior cells; its
        # ghost cells are multigrid scratch
        compare(sim, run, cc_vars=[0, 1, 2, 3, 4, 6, 7, 8], where=op)
        from parity import interior_mask
        m = interior_mask(sim.meta(), cfg.box_size)
        assert np.array_equal(sim.cc(5)[m], run.cc(5)[m])
        return
    elif op == "gc":
        sim.op("gc_tree", 0, 0); run.gc_tree(0, 0)
    elif op == "restrict":
        sim.op("restrict_tree", 1); run.restrict_tree(1)
    elif op == "fld_from_pot":
        sim.op("fld_from_pot"); run.fld_from_pot()
    compare(sim, run, where=op)


def test_grid_photoionization_step():
    cfg = config.cylindrical_16mm(photoi=True, photoi_team=1000)
    sim = a5ref.Sim(cfg, n_threads=4)
    sim.init()
    run = device_from_oracle(sim, cfg)
    dist, frac, _ = sim.photon_table()
    run.set_photon_table(dist, frac)
    run.set_rng_state(sim.rng_state())
    run.set_ctas(32)
    for k in range(2):
        dt = sim.get_max_dt()
        sim.step(dt)
        run.step(dt)
        compare(sim, run, where=f"photoionization grid step {k}")
        assert np.array_equal(sim.rng_state(), run.rng_state())


def test_grid_mixed_matches_one_block():
    """The mixed form in grid mode (FP32 correction solve in device memory)
    gives exactly what one block gives."""
    cfg = config.cartesian_8mm()
    sim = _oracle(cfg)
    a = device_from_oracle(sim, cfg)
    b = device_from_oracle(sim, cfg)
    for r in (a, b):
        r.set_precision(True, (0, 2, 2, 8, 2))
    b.set_ctas(24)
    dt = sim.get_max_dt()
    for _ in range(3):
        a.step(dt)
        b.step(dt)
    for iv in (dv.I_ELEC, dv.I_PION, dv.I_PHI, dv.I_FLD):
        assert np.array_equal(a.cc(iv), b.cc(iv)), iv


def test_grid_driver_run():
    """The product's driver in grid mode (steps, reductions, flags, regrid
    prolongation, field solves all on 8 blocks) against the oracle."""
    cfg = config.cartesian_8mm(applied_fld=7e6, lvls_max=6)
    sim = streamer.Simulation(cfg)
    sim.device.set_ctas(8)
    ref = a5ref.Sim(cfg, n_threads=4)
    assert sim.init() == ref.init()
    for k in range(6):
        assert sim.advance(True) == ref.advance(True)
        meta, _, _ = sim.tree.export()
        assert np.array_equal(meta, ref.meta())
        m = side_mask(meta, cfg.box_size)
        for iv in (0, 1, 4, 5):
            assert np.array_equal(sim.device.cc(iv)[m], ref.cc(iv)[m]), (k, iv)


def test_grid_uniform_large_tree():
    """A uniformly refined mesh (65,536 leaf cells at level 4 of the 8 mm
    case): the whole GPU's blocks against the oracle over a step."""
    cfg = config.cartesian_uniform(4)
    sim = a5ref.Sim(cfg, n_threads=8)
    sim.init()
    assert sim.n_leaf_cells() == (32 * 8) ** 2
    run = device_from_oracle(sim, cfg)
    run.set_ctas(run.ctas()[1])
    run.set_grid_local(4096)
    dt = sim.get_max_dt()
    assert run.get_max_dt() == dt
    sim.step(dt)
    run.step(dt)
    compare(sim, run, where="uniform level 4")


def test_grid_barrier_timeout_is_reported_and_recoverable():
    cfg = config.cartesian_8mm()
    sim = _oracle(cfg, blocks=1)
    run = device_from_oracle(sim, cfg)
    dt = sim.get_max_dt()
    run.set_ctas(4, 0)            # every barrier wait runs out at once
    run.step(dt)
    with pytest.raises(_lib.A5GError) as e:
        run.sync()
    assert e.value.code == _lib.A5G_TIMEOUT
    # the context stays usable: restore the state, default budget, step again
    run.set_ctas(4)
    device_from_oracle(sim, cfg, run)
    sim.step(dt)
    run.step(dt)
    compare(sim, run, where="after a timeout")


def test_set_ctas_rejects_too_many():
    cfg = config.cartesian_8mm()
    run = dv.DeviceRun(cfg)
    _, most = run.ctas()
    assert most >= 148
    with pytest.raises(_lib.A5GError):
        run.set_ctas(most + 1)
    with pytest.raises(_lib.A5GError):
        run.set_ctas(0)
