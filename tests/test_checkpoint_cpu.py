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
