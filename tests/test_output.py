"""VTK output of the leaf cells (a$D_write_vtk layout), written from arrays in
the device layout -- here the oracle's state of the 8 mm case -- and read back."""
import numpy as np

import a5ref
from a5_streamer_b200 import config, output


def _state():
    cfg = config.cartesian_8mm()
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    return cfg, sim


def test_vtk_round_trip(tmp_path):
    cfg, sim = _state()
    meta, geom, levels = sim.meta(), sim.geom(), sim.levels()
    path = output.write_vtk(str(tmp_path / "run"), meta, geom, levels,
                            {"e": sim.cc(0), "phi": sim.cc(4)}, time=1.5e-9, n_cycle=7)
    assert path.endswith(".vtu")
    d = output.read_vtk(path)
    mesh = output.leaf_mesh(meta, geom, levels)
    nc = cfg.box_size
    n_leaf_boxes = sum(len(levels[l][1]) for l in levels if l >= 1)
    assert mesh["n_boxes"] == n_leaf_boxes
    assert d["Points"].shape == (n_leaf_boxes * (nc + 1) ** 2, 3)
    assert len(d["types"]) == sim.n_leaf_cells() and set(d["types"]) == {output.VTK_PIXEL}
    assert np.array_equal(d["offsets"], 4 * np.arange(1, sim.n_leaf_cells() + 1))
    assert d["TIME"][0] == 1.5e-9 and d["CYCLE"][0] == 7
    # every cell's four nodes span one cell of its box
    pts = d["Points"][:, :2].astype(np.float64)
    con = d["connectivity"].reshape(-1, 4)
    dx = pts[con[:, 1], 0] - pts[con[:, 0], 0]
    dy = pts[con[:, 2], 1] - pts[con[:, 0], 1]
    drs = geom[mesh["box"], 3]
    assert np.allclose(dx, drs, rtol=1e-6) and np.allclose(dy, drs, rtol=1e-6)
    assert pts[:, 0].min() == 0.0 and abs(pts[:, 0].max() - cfg.domain_len[0]) < 1e-9
    # values are the leaf cells' values, exactly
    e = sim.cc(0)
    assert np.array_equal(d["e"], e[mesh["box"], mesh["slot"]])
    # leaf cells cover the domain once
    area = float(np.sum(drs ** 2))
    assert abs(area - cfg.domain_len[0] * cfg.domain_len[1]) < 1e-12


def test_face_means_and_axis_profile():
    cfg, sim = _state()
    meta, geom, levels = sim.meta(), sim.geom(), sim.levels()
    mesh = output.leaf_mesh(meta, geom, levels)
    fx, fy = sim.fc(0, 1), sim.fc(1, 1)
    mx, my = output.face_means(mesh, fx, fy)
    k = 5
    b, s, nc = mesh["box"][k], mesh["slot"][k], cfg.box_size
    i, j = s % (nc + 2), s // (nc + 2)
    assert mx[k] == 0.5 * (fx[b, (i - 1) + (nc + 1) * (j - 1)] + fx[b, i + (nc + 1) * (j - 1)])
    assert my[k] == 0.5 * (fy[b, (i - 1) + nc * (j - 1)] + fy[b, (i - 1) + nc * j])
    z, f, n = output.axis_profile(sim.cc(5), sim.cc(0), meta, geom, levels, cfg)
    assert np.all(np.diff(z) >= 0) and len(z) == len(f) == len(n) > 0


def test_vtk_matches_the_reference_layout(tmp_path):
    """The file output.write_vtk writes against the oracle's restatement of
    the arrays a$D_write_vtk builds (afivo/src/m_aX_io.f90:20-207): the same
    node coordinates (stored as Float32, as m_vtk.f90 writes them), the same
    pixel connectivity, offsets and types, and the same cell values and face
    means in the same order, to the bit."""
    cfg = config.cylindrical_16mm()
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    for _ in range(2):
        sim.advance(True)
    meta, geom, levels = sim.meta(), sim.geom(), sim.levels()
    mesh = output.leaf_mesh(meta, geom, levels)
    mx, my = output.face_means(mesh, sim.fc(0, 1), sim.fc(1, 1))
    path = output.write_vtk(str(tmp_path / "ref"), meta, geom, levels,
                            {"n_e": sim.cc(0), "phi": sim.cc(4), "fld_x": mx, "fld_y": my})
    d = output.read_vtk(path)
    ref = sim.vtk_arrays([a5ref.I_ELEC, a5ref.I_PHI], [a5ref.F_FLD])
    assert np.array_equal(d["Points"][:, :2], ref["coords"].astype(np.float32))
    assert np.all(d["Points"][:, 2] == 0)
    assert np.array_equal(d["connectivity"], ref["connectivity"])
    assert np.array_equal(d["offsets"], ref["offsets"])
    assert np.array_equal(d["types"], ref["types"])
    for k, name in enumerate(("n_e", "phi", "fld_x", "fld_y")):
        assert np.array_equal(d[name], ref["values"][k]), name
