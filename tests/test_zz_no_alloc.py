"""a5g_step_batch_static: the batched step for callers that cannot allocate
device memory while stepping (a host with a device-memory budget fixed before
the time loop, or a stepping path that must not block on the allocator).

Through the C ABI, two calls in a row of the allocation-free entry point must
give exactly (bit for bit, the tolerance of the other parity tests) what two
calls of a5g_step_batch give on identical inputs, for FP64 members, for
members with Monte Carlo photoionization (whose photon pass rewrites the
shared descriptor table before the step pass) and for mixed-precision
members; the FP64 members also match the oracle directly. Every member is
read through its own stream right after the calls, without a wait on the
first member: the batch is ordered before the members' later work on the
device. Runs standalone in a fresh process as well as after the other
tests."""
import ctypes

import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import _lib, config
from parity import compare, device_from_oracle

pytestmark = pytest.mark.gpu


def _member(cfg, sim, mixed=False):
    run = device_from_oracle(sim, cfg)
    if cfg.photoi_enabled:
        dist, frac, _ = sim.photon_table()
        run.set_photon_table(dist, frac)
        run.set_rng_state(sim.rng_state())
    if mixed:
        run.set_precision(True, (0, 2, 2, 4, 2))
    return run


def _state(run):
    cc = [run.cc(iv) for iv in range(9)]
    fc = [run.fc(d, f) for d in range(2) for f in range(2)]
    return cc + fc


def _call(name, runs, dts):
    arr = (ctypes.c_void_p * len(runs))(*[r.h.value for r in runs])
    d = np.ascontiguousarray(dts, dtype=np.float64)
    _lib.call(name, arr, len(runs), d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))


def _oracles(cfgs):
    sims = []
    for cfg in cfgs:
        sim = a5ref.Sim(cfg, n_threads=2)
        sim.init()
        sim.advance(True)
        sims.append(sim)
    return sims


@pytest.mark.parametrize("kind", ["fp64", "photoionization", "mixed"])
def test_static_batch_matches_batch(kind):
    if kind == "photoionization":
        cfgs = [config.cylindrical_16mm(photoi=True, photoi_team=512),
                config.cylindrical_16mm(photoi=True, photoi_team=2000, rng_seed=(1, 2, 3, 4)),
                config.cylindrical_16mm()]
    else:
        cfgs = [config.cartesian_8mm(), config.cylindrical_16mm(), config.cartesian_8mm()]
    sims = _oracles(cfgs)
    mixed = kind == "mixed"
    a = [_member(c, s, mixed and k != 1) for k, (c, s) in enumerate(zip(cfgs, sims))]
    b = [_member(c, s, mixed and k != 1) for k, (c, s) in enumerate(zip(cfgs, sims))]
    base = [s.get_max_dt() for s in sims]
    for step in range(2):
        dts = [dt * (1.0 - 0.25 * step) for dt in base]
        _call("a5g_step_batch", a, dts)
        _call("a5g_step_batch_static", b, dts)
        if not mixed:
            for s, dt in zip(sims, dts):
                s.step(dt)
    # no sync of member 0 first: each read below is queued on the member's
    # own stream, which the batch call ordered after the batch
    for ra, rb in zip(a[::-1], b[::-1]):
        for xa, xb in zip(_state(ra), _state(rb)):
            assert np.array_equal(xa, xb)
    if not mixed:
        for s, rb in zip(sims, b):
            compare(s, rb, where=f"static batch ({kind})")
            if s.cfg.photoi_enabled:
                assert np.array_equal(s.rng_state(), rb.rng_state())
    # the result is a real step: it moved the densities
    assert not np.array_equal(_state(b[0])[0], sims[0].cc(0) if mixed else _oracles(cfgs[:1])[0].cc(0))


def test_static_batch_rejects_oversize():
    cfg = config.cartesian_8mm()
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    run = device_from_oracle(sim, cfg)
    n = 1025
    arr = (ctypes.c_void_p * n)(*([run.h.value] * n))
    d = np.full(n, 1e-12)
    code = _lib.lib().a5g_step_batch_static(arr, n, d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert code == _lib.A5G_EINVAL
    assert b"A5G_STATIC_BATCH_MAX" in _lib.lib().a5g_last_error()


def test_static_batch_refuses_unsized_fp32_storage():
    """A mixed member whose tree is not staged in shared memory keeps FP32
    arrays in device memory, sized to its box storage. When a tree upload
    grows that storage, the allocation-free call does not allocate new
    arrays: it refuses the member until one ordinary step has sized them,
    and then gives what a5g_step_batch gives."""
    cfg = config.cartesian_8mm()
    small = a5ref.Sim(cfg, n_threads=2)
    small.init()
    big_cfg = config.cartesian_uniform(4)
    big = a5ref.Sim(big_cfg, n_threads=2)
    big.init()
    runs = []
    for _ in range(2):
        r = _member(cfg, small, mixed=True)
        _lib.call("a5g_debug_set_staging", r.h, 0)   # FP32 arrays in device memory
        device_from_oracle(big, big_cfg, r)          # grows the box storage
        runs.append(r)
    a, b = runs
    dt = [big.get_max_dt()]
    arr = (ctypes.c_void_p * 1)(b.h.value)
    d = np.ascontiguousarray(dt, dtype=np.float64)
    code = _lib.lib().a5g_step_batch_static(arr, 1, d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert code == _lib.A5G_ESTATE
    assert b"FP32 storage" in _lib.lib().a5g_last_error()
    _call("a5g_step_batch", [a], dt)
    _call("a5g_step_batch", [b], dt)     # sizes b's FP32 arrays
    _call("a5g_step_batch", [a], dt)
    _call("a5g_step_batch_static", [b], dt)
    for xa, xb in zip(_state(a), _state(b)):
        assert np.array_equal(xa, xb)
