"""Run checkpoints on the CPU: the oracle writes its state in the layout of
the product's a5s_checkpoint_save and resumes from such a buffer. A resumed
oracle run continues exactly as the uninterrupted one -- step sizes, regrids
(refinement and derefinement), generator draws, every cell value -- which
pins the layout's contents: a checkpoint holds all the state the next block
reads. (The device writes the same layout: tests/test_gpu_checkpoint.py.)"""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config
from parity import side_mask

CASES = {
    "cart": (config.cartesian_8mm(), 2, 3),
    "cyl_photoi": (config.cylindrical_16mm(photoi=True), 2, 3),
    "cart_active": (config.cartesian_8mm(applied_fld=7e6, lvls_max=6), 4, 6),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_resumes_from_its_checkpoint(name):
    cfg, first, then = CASES[name]
    a = a5ref.Sim(cfg, n_threads=2)
    a.init()
    for _ in range(first):
        a.advance(True)
    ck = a.checkpoint()
    dts_a = [a.advance(True) for _ in range(then)]

    b = a5ref.Sim(cfg, n_threads=2)  # fresh: base mesh only
    b.load_checkpoint(ck)
    assert b.checkpoint() == ck
    dts_b = [b.advance(True) for _ in range(then)]
    assert dts_a == dts_b
    assert a.time == b.time
    meta = a.meta()
    assert np.array_equal(meta, b.meta())
    assert np.array_equal(a.geom(), b.geom())
    la, lb = a.levels(), b.levels()
    assert sorted(la) == sorted(lb)
    for lvl in la:
        for x, y in zip(la[lvl], lb[lvl]):
            assert np.array_equal(x, y), lvl
    m = side_mask(meta, cfg.box_size)
    for iv in range(9):
        assert np.array_equal(a.cc(iv)[m], b.cc(iv)[m]), iv
    if cfg.photoi_enabled:
        assert np.array_equal(a.rng_state(), b.rng_state())


def test_malformed_checkpoints_are_rejected():
    cfg = config.cartesian_8mm()
    a = a5ref.Sim(cfg, n_threads=2)
    a.init()
    ck = a.checkpoint()
    b = a5ref.Sim(cfg, n_threads=2)
    with pytest.raises(ValueError):
        b.load_checkpoint(b"XXXX" + ck[4:])
    with pytest.raises(ValueError):
        b.load_checkpoint(ck + b"\0" * 8)


def test_host_reader_gives_the_run_state(tmp_path):
    """a5_streamer_b200.checkpoint reads a checkpoint on the host into the
    package's formats: the tree as Tree.export gives it, the cell and face
    variables in the download layout, time and generator state."""
    from a5_streamer_b200 import checkpoint
    cfg = config.cylindrical_16mm(photoi=True)
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    sim.advance(True)
    path = tmp_path / "run.a5ck"
    path.write_bytes(sim.checkpoint())
    ck = checkpoint.load(str(path))
    assert ck.time == sim.time and np.array_equal(ck.rng, sim.rng_state())
    assert (ck.min_lvl, ck.max_lvl, ck.max_id) == (sim.min_lvl, sim.max_lvl, sim.max_id)
    assert ck.coord == 1 and ck.photoionization and ck.box_size == cfg.box_size
    assert np.array_equal(ck.meta, sim.meta()) and np.array_equal(ck.geom, sim.geom())
    rl = sim.levels()
    assert sorted(ck.levels) == sorted(rl)
    for lvl in rl:
        for x, y in zip(ck.levels[lvl], rl[lvl]):
            assert np.array_equal(x, y)
    for iv in range(9):
        assert np.array_equal(ck.cc[iv], sim.cc(iv)), iv
    for d in range(2):
        for f in range(2):
            assert np.array_equal(ck.fc[2 * d + f], sim.fc(d, f))
    assert ck.n_leaf_cells() == sim.n_leaf_cells()


def test_vtk_from_a_checkpoint_equals_the_live_output(tmp_path):
    from a5_streamer_b200 import checkpoint, output
    cfg = config.cartesian_8mm()
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    sim.advance(True)
    path = tmp_path / "run.a5ck"
    path.write_bytes(sim.checkpoint())
    a = checkpoint.write_vtk(str(path), str(tmp_path / "from_ck"))
    b = output.write_state(str(tmp_path / "live"), sim.meta(), sim.geom(), sim.levels(),
                           sim.cc, sim.fc, sim.time)
    assert open(a, "rb").read() == open(b, "rb").read()


def test_host_reader_rejects_malformed_buffers():
    from a5_streamer_b200 import checkpoint
    cfg = config.cartesian_8mm()
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    ck = sim.checkpoint()
    for bad in (b"", ck[:40], b"XXXX" + ck[4:], ck[:-8], ck + b"\0" * 8):
        with pytest.raises(ValueError):
            checkpoint.read(bad)


def test_host_reader_and_library_agree_on_the_header():
    """The magic and version the host reader expects are the library's."""
    import os
    import re
    from a5_streamer_b200 import checkpoint
    src = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                            "a5_streamer_b200", "csrc", "host.cpp")).read()
    magic = int(re.search(r"kCkMagic = (0x[0-9A-Fa-f]+)u", src).group(1), 16)
    version = int(re.search(r"kCkVersion = (\d+)", src).group(1))
    assert (magic, version) == (checkpoint.MAGIC, checkpoint.VERSION)
    assert (magic, version) == (a5ref.Sim._CK_MAGIC, a5ref.Sim._CK_VERSION)
