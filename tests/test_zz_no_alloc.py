"""a5g_step_batch_static: the batched step for callers that cannot allocate
device memory while stepping (a host with a device-memory budget fixed before
the time loop, or a stepping path that must not block on the allocator).

Through the C ABI, two calls in a row of the allocation-free entry point must
give exactly (bit for bit, the tolerance of the other parity tests) what two
calls of a5g_step_batch give on identical inputs. Runs standalone in a fresh
process as well as after the other tests."""
import ctypes

import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import _lib, config
from a5_streamer_b200 import device as dv
from parity import device_from_oracle

pytestmark = pytest.mark.gpu


def _runs(cfg, sim, n):
    return [device_from_oracle(sim, cfg) for _ in range(n)]


def _state(run):
    cc = [run.cc(iv) for iv in range(9)]
    fc = [run.fc(d, f) for d in range(2) for f in range(2)]
    return cc + fc


def _call(name, runs, dts):
    arr = (ctypes.c_void_p * len(runs))(*[r.h.value for r in runs])
    d = np.ascontiguousarray(dts, dtype=np.float64)
    _lib.call(name, arr, len(runs), d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))


@pytest.mark.parametrize("make_cfg", [config.cartesian_8mm, config.cylindrical_16mm])
def test_static_batch_matches_batch(make_cfg):
    cfg = make_cfg()
    sim = a5ref.Sim(cfg, n_threads=2)
    sim.init()
    sim.advance(True)
    dt = sim.get_max_dt()
    a = _runs(cfg, sim, 3)
    b = _runs(cfg, sim, 3)
    dts = [dt, 0.5 * dt, 0.25 * dt]
    for _ in range(2):
        _call("a5g_step_batch", a, dts)
        _call("a5g_step_batch_static", b, dts)
    a[0].sync()
    b[0].sync()
    for ra, rb in zip(a, b):
        for xa, xb in zip(_state(ra), _state(rb)):
            assert np.array_equal(xa, xb)
    # the result is a real step: it moved the densities
    assert not np.array_equal(_state(a[0])[0], sim.cc(0))


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
