"""VTK output of a device-resident run."""
import numpy as np
import pytest

from a5_streamer_b200 import config, output, streamer

pytestmark = pytest.mark.gpu


def test_write_run(tmp_path):
    cfg = config.cylindrical_16mm()
    sim = streamer.Simulation(cfg)
    sim.init()
    sim.advance(True)
    path = output.write_run(str(tmp_path / "cyl"), sim, n_cycle=1)
    d = output.read_vtk(path)
    meta, geom, levels = sim.tree.export()
    mesh = output.leaf_mesh(meta, geom, levels)
    assert len(d["types"]) == sim.device.n_leaf_cells()
    assert np.array_equal(d["phi"], sim.device.cc(4)[mesh["box"], mesh["slot"]])
    assert np.array_equal(d["fld"], sim.device.cc(5)[mesh["box"], mesh["slot"]])
    assert d["TIME"][0] == sim.time and "flux_x" in d and np.isfinite(d["flux_y"]).all()


def test_run_properties():
    from a5_streamer_b200 import diagnostics
    cfg = config.cylindrical_16mm()
    sim = streamer.Simulation(cfg)
    sim.init()
    sim.advance(True)
    props, axis = diagnostics.run_properties(sim)
    assert len(props) == 39 and props["E_bg"] == cfg.applied_fld
    assert props["Ez_max"] > cfg.applied_fld and 0 < props["Er_max(z)"] < cfg.domain_len_z
    assert axis.shape[0] == 5 and np.all(np.diff(axis[0]) > 0)
