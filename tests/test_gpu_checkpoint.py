"""Checkpoint / resume (include/a5t.h a5s_checkpoint_*): a run resumed from a
checkpoint, on a fresh run of the same configuration, continues exactly as
the run that wrote it -- same step sizes, same regrids, the same state to
the bit -- and equals the oracle's uninterrupted run. Bad buffers and
checkpoints of another configuration are rejected and leave the run as it
was."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import _lib, config, streamer

pytestmark = pytest.mark.gpu


def _state(sim):
    meta, geom, levels = sim.tree.export()
    cc = [sim.device.cc(iv) for iv in range(9)]
    fc = [sim.device.fc(d, f) for d in range(2) for f in range(2)]
    rng = sim.device.rng_state() if sim.cfg.photoi_enabled else None
    return meta, geom, levels, cc, fc, rng


def _assert_same(a, b, where):
    ma, ga, la, ca, fa, ra = a
    mb, gb, lb, cb, fb, rb = b
    assert np.array_equal(ma, mb), f"{where}: topology differs"
    assert np.array_equal(ga, gb), f"{where}: geometry differs"
    assert la.keys() == lb.keys()
    for lvl in la:
        for x, y in zip(la[lvl], lb[lvl]):
            assert np.array_equal(x, y), f"{where}: level lists differ at level {lvl}"
    used = ma[:, 0] == 1
    for iv, (x, y) in enumerate(zip(ca, cb)):
        assert np.array_equal(x[used], y[used]), f"{where}: cell variable {iv} differs"
    for k, (x, y) in enumerate(zip(fa, fb)):
        assert np.array_equal(x[used], y[used]), f"{where}: face variable {k} differs"
    if ra is not None:
        assert np.array_equal(ra, rb), f"{where}: generator state differs"


@pytest.mark.parametrize("name,first,then", [
    ("cartesian_8mm", 3, 4),
    ("cylindrical_16mm_photoi", 3, 4),
    # refinement and derefinement after the resume
    ("cartesian_active", 4, 8),
])
def test_resume_continues_bit_for_bit(name, first, then, tmp_path):
    cfg = {"cartesian_8mm": config.cartesian_8mm(),
           "cylindrical_16mm_photoi": config.cylindrical_16mm(photoi=True),
           "cartesian_active": config.cartesian_8mm(applied_fld=7e6, lvls_max=6)}[name]
    a = streamer.Simulation(cfg)
    a.init()
    for _ in range(first):
        a.advance(True)
    path = tmp_path / "run.a5ck"
    a.save(str(path))
    t_ck = a.time
    dts_a = [a.advance(True) for _ in range(then)]
    end_a = _state(a)

    b = streamer.Simulation(cfg)  # fresh: base mesh only, never initialised
    b.load(str(path))
    assert b.time == t_ck
    dts_b = [b.advance(True) for _ in range(then)]
    assert dts_a == dts_b
    assert a.time == b.time
    _assert_same(end_a, _state(b), "resumed")

    # a second checkpoint of the resumed run equals the first run's
    assert a.checkpoint() == b.checkpoint()


def test_resumed_run_equals_the_oracle_uninterrupted():
    cfg = config.cartesian_8mm()
    a = streamer.Simulation(cfg)
    a.init()
    a.advance(True)
    a.advance(True)
    ck = a.checkpoint()
    a.close()
    b = streamer.Simulation(cfg)
    b.restore(ck)
    ref = a5ref.Sim(cfg, n_threads=4)
    ref.init()
    ref.advance(True)
    ref.advance(True)
    for k in range(3):
        assert b.advance(True) == ref.advance(True), k
    assert b.time == ref.time
    meta, geom, _ = b.tree.export()
    assert np.array_equal(meta, ref.meta())
    assert np.array_equal(geom, ref.geom())
    used = meta[:, 0] == 1
    for iv in (0, 1, 4):
        x, y = b.device.cc(iv), ref.cc(iv)
        n = cfg.box_size
        g = n + 2
        for id_ in np.nonzero(used)[0]:
            nn = meta[id_, 14]
            gg = nn + 2
            xi = x[id_, :gg * gg].reshape(gg, gg)[1:nn + 1, 1:nn + 1]
            yi = y[id_, :gg * gg].reshape(gg, gg)[1:nn + 1, 1:nn + 1]
            assert np.array_equal(xi, yi), (iv, id_)
        assert g == 10


def test_bad_checkpoints_are_rejected_and_change_nothing():
    cfg = config.cartesian_8mm()
    a = streamer.Simulation(cfg)
    a.init()
    a.advance(True)
    ck = a.checkpoint()
    before = _state(a)
    t0 = a.time
    # a box record whose level disagrees with its level list (header 80
    # bytes, then 80-byte records per id; the level is the record's second int)
    import struct
    off = 80 + 80 * 1 + 4
    (lvl,) = struct.unpack_from("<i", ck, off)
    relevelled = ck[:off] + struct.pack("<i", lvl + 1) + ck[off + 4:]
    for bad in (b"", ck[:10], ck[:len(ck) // 2], ck + b"\0", b"XXXX" + ck[4:], relevelled):
        with pytest.raises(_lib.A5GError) as e:
            a.restore(bad)
        assert e.value.code == _lib.A5G_EINVAL
    # a run of another configuration (different applied field)
    other = streamer.Simulation(config.cartesian_8mm(applied_fld=3e6))
    other.init()
    with pytest.raises(_lib.A5GError) as e:
        a.restore(other.checkpoint())
    assert e.value.code == _lib.A5G_EINVAL and "configuration" in str(e.value)
    assert a.time == t0
    _assert_same(before, _state(a), "after rejected loads")
    # the untouched run still steps as before
    c = streamer.Simulation(cfg)
    c.restore(ck)
    assert a.advance(True) == c.advance(True)


def test_layout_is_the_documented_one():
    """The buffer parses with the layout written out beside a5s_checkpoint_*
    (native byte order, no padding), and its parts are the run's own tree,
    time and cell data."""
    import struct
    cfg = config.cylindrical_16mm(photoi=True)
    sim = streamer.Simulation(cfg)
    sim.init()
    sim.advance(True)
    ck = sim.checkpoint()
    magic, version, _fp = struct.unpack_from("<IIQ", ck, 0)
    assert magic == 0x4B433541 and version == 1
    off = 16
    (nc, coord, lvls_max, min_lvl, max_lvl, max_id, n_lists, cslot, fslot, photoi) = \
        struct.unpack_from("<10i", ck, off)
    off += 40
    (t,) = struct.unpack_from("<d", ck, off)
    off += 8
    rng = np.frombuffer(ck, dtype="<i4", count=4, offset=off)
    off += 16
    assert (nc, coord, photoi) == (8, 1, 1) and cslot == 100 and fslot == 72
    assert t == sim.time and np.array_equal(rng, sim.device.rng_state())
    assert (min_lvl, max_lvl, max_id) == (sim.tree.min_lvl, sim.tree.max_lvl, sim.tree.max_id)
    rec = np.dtype([("i", "<i4", 14), ("d", "<f8", 3)])
    recs = np.frombuffer(ck, dtype=rec, count=max_id + 1, offset=off)
    off += rec.itemsize * (max_id + 1)
    meta, geom, levels = sim.tree.export()
    used = meta[:, 0] == 1
    assert np.array_equal(recs["i"][1:, 0], meta[1:, 0])            # in_use
    ri, rd = recs["i"][used], recs["d"][used]
    assert np.array_equal(ri[:, 1], meta[used, 1])                  # level
    assert np.array_equal(ri[:, 4], meta[used, 5])                  # parent
    assert np.array_equal(ri[:, 5], meta[used, 14])                 # cells per edge
    assert np.array_equal(ri[:, 6:10], meta[used, 6:10])            # children
    assert np.array_equal(ri[:, 10:14], meta[used, 10:14])          # neighbours
    assert np.array_equal(rd[:, 0], geom[used, 3])                  # dr
    for k in range(n_lists):
        a, b, c = struct.unpack_from("<3i", ck, off)
        off += 12
        lst = np.frombuffer(ck, dtype="<i4", count=a + b + c, offset=off)
        off += 4 * (a + b + c)
        lvl = min_lvl + k
        if lvl in levels:
            ids, leaves, parents = levels[lvl]
            assert np.array_equal(lst[:a], ids) and np.array_equal(lst[a:a + b], leaves)
            assert np.array_equal(lst[a + b:], parents)
    cc = np.frombuffer(ck, dtype="<f8", count=9 * (max_id + 1) * cslot, offset=off)
    off += 8 * cc.size
    for iv in range(9):
        x = cc[iv * (max_id + 1) * cslot:(iv + 1) * (max_id + 1) * cslot].reshape(max_id + 1, cslot)
        assert np.array_equal(x[used], sim.device.cc(iv)[used]), iv
    off += 8 * 2 * 2 * (max_id + 1) * fslot
    assert off == len(ck)
