"""Dielectric runs (eps != 1 in the bottom quarter of the domain, set per box
as set_box_eps does): the multigrid tags each box from its eps
(mg$D_set_box_tag) and applies the eps operators (gsrb_lpld / lpld /
corr_lpld, cylindrical clpld / gsrb_clpld) to the dielectric boxes. Device
against oracle, bit for bit, per operation and over whole driver runs."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config, streamer
from a5_streamer_b200 import device as dv
from parity import compare, device_from_oracle, side_mask, interior_mask

pytestmark = pytest.mark.gpu

CASES = {
    "cart": config.cartesian_8mm(epsilon_diel=2.0),
    "cyl": config.cylindrical_16mm(epsilon_diel=3.0),
}
DT = 2.5e-11


def _oracle(cfg, blocks=2):
    sim = a5ref.Sim(cfg, n_threads=4)
    sim.init()
    for _ in range(blocks):
        sim.advance(True)
    return sim


@pytest.mark.parametrize("name", sorted(CASES))
def test_diel_operations(name):
    cfg = CASES[name]
    sim = _oracle(cfg)
    run = device_from_oracle(sim, cfg)
    compare(sim, run, where="upload")
    sim.op("compute_fld", 0)
    run.compute_fld(False)
    compare(sim, run, where="compute_fld")
    sim.op("fmg", 0, 1)
    run.fas_fmg(False, True)
    compare(sim, run, cc_vars=[0, 1, 2, 3, 4, 6, 7, 8], where="first FMG")
    for k in range(3):
        sim.step(DT)
        run.step(DT)
        compare(sim, run, where=f"step {k}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_diel_driver_matches_oracle(name):
    cfg = CASES[name]
    sim = streamer.Simulation(cfg)
    ref = a5ref.Sim(cfg, n_threads=4)
    assert sim.init() == ref.init()
    for k in range(6):
        assert sim.advance(True) == ref.advance(True), k
        meta, geom, levels = sim.tree.export()
        assert np.array_equal(meta, ref.meta()), f"block {k}: topology differs"
        m = side_mask(meta, cfg.box_size)
        for iv in (0, 1, 4, 5, 8):
            assert np.array_equal(sim.device.cc(iv)[m], ref.cc(iv)[m]), f"block {k}: variable {iv}"


def test_diel_eps_operators_matter():
    """The eps operators change the solution: the same state solved with eps
    uploaded as 1 everywhere differs from the dielectric solve."""
    cfg = CASES["cart"]
    sim = _oracle(cfg)
    run = device_from_oracle(sim, cfg)
    plain = device_from_oracle(sim, cfg)
    plain.set_cc(dv.I_EPS, np.ones_like(sim.cc(dv.I_EPS)))
    for r in (run, plain):
        r.compute_fld(False)
    mi = interior_mask(sim.meta(), cfg.box_size)
    assert not np.array_equal(run.cc(dv.I_PHI)[mi], plain.cc(dv.I_PHI)[mi])


def test_mixed_form_rejects_dielectric_runs():
    run = dv.DeviceRun(CASES["cart"])
    with pytest.raises(Exception):
        run.set_precision(True)
