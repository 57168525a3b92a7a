"""The oracle (CPU) and the device path (GPU) against the committed golden
fixtures of tests/golden/ (generated by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import a5ref
from make_golden import CASES, VARS, interiors

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(HERE, f"{name}_2blocks.npz"))


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_golden(name):
    g = _load(name)
    cfg = CASES[name]()
    sim = a5ref.Sim(cfg, n_threads=3)
    assert sim.init() == int(g["n_init"])
    dts = [sim.advance(True) for _ in range(2)]
    assert np.array_equal(np.asarray(dts), g["dts"])
    meta = sim.meta()
    assert np.array_equal(meta, g["meta"])
    for iv in VARS:
        assert np.array_equal(interiors(meta, sim.cc(iv), cfg.box_size), g[f"v{iv}"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_device_reproduces_golden(name):
    from a5_streamer_b200 import streamer
    g = _load(name)
    cfg = CASES[name]()
    sim = streamer.Simulation(cfg)
    assert sim.init() == int(g["n_init"])
    dts = [sim.advance(True) for _ in range(2)]
    assert np.array_equal(np.asarray(dts), g["dts"])
    meta, _, _ = sim.tree.export()
    assert np.array_equal(meta, g["meta"])
    for iv in VARS:
        assert np.array_equal(interiors(meta, sim.device.cc(iv), cfg.box_size), g[f"v{iv}"])
    assert np.array_equal(sim.device.dt_reductions(), g["dt_red"])
