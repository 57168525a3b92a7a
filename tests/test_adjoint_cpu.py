"""The linear phases the device adjoint transposes (a5a_debug_tape, built on
the host without a GPU): applied forward they reproduce the oracle's
operations on the 8 mm mesh, and their transposed application passes the
dot-product test <T x, y> = <x, T^t y>."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import adjoint, config

SLOT, FSLOT, NVC = 100, 72, 9
SEG = dict(copy=0, cons=1, rstr=2, rhs=3, fmg=4, fmg1=5, faces=6, gcfld=7, avg=8)


@pytest.fixture(scope="module")
def mesh():
    cfg = config.cartesian_8mm()
    s = a5ref.Sim(cfg, n_threads=4)
    s.init()
    dt = s.get_max_dt()
    s.step(dt)  # a state with a nonzero previous potential and fluxes
    meta, geom, levels = s.meta(), s.geom(), s.levels()
    cap = meta.shape[0]
    tapes = {k: adjoint.debug_tape(meta, geom, levels, cap, cfg.n_cycle_base, v)
             for k, v in SEG.items()}
    return s, cfg, cap, tapes


def state(s, cap, n):
    x = np.zeros(n)
    m = s.max_id + 1
    for iv in range(NVC):
        x[iv * cap * SLOT:(iv + 1) * cap * SLOT].reshape(cap, SLOT)[:m] = s.cc(iv)
    base = NVC * cap * SLOT
    for d in range(2):
        for f in range(2):
            o = base + (2 * d + f) * cap * FSLOT
            x[o:o + cap * FSLOT].reshape(cap, FSLOT)[:m] = s.fc(d, f)
    x[n - 1] = s.applied_voltage
    return x


def forward(tape, x):
    pr, rd, rs, rt, ts, tc, _ = tape
    x = x.copy()
    row_of = np.repeat(np.arange(len(rd)), np.diff(rt))
    contrib = np.zeros(len(rd))
    for p in range(len(pr) - 1):
        r0, r1 = pr[p], pr[p + 1]
        t0, t1 = rt[r0], rt[r1]
        contrib[r0:r1] = 0
        np.add.at(contrib, row_of[t0:t1], tc[t0:t1] * x[ts[t0:t1]])
        x[rd[r0:r1]] = rs[r0:r1] * x[rd[r0:r1]] + contrib[r0:r1]
    return x


def transpose(tape, y):
    pr, rd, rs, rt, ts, tc, _ = tape
    y = y.copy()
    row_of = np.repeat(np.arange(len(rd)), np.diff(rt))
    for p in range(len(pr) - 2, -1, -1):
        r0, r1 = pr[p], pr[p + 1]
        t0, t1 = rt[r0], rt[r1]
        lam = y[rd[r0:r1]].copy()
        y[rd[r0:r1]] = rs[r0:r1] * lam
        np.add.at(y, ts[t0:t1], tc[t0:t1] * lam[row_of[t0:t1] - r0])
    return y


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("first", [False, True])
def test_fmg_phases_reproduce_the_oracle(mesh, first):
    s, cfg, cap, tapes = mesh
    s.op("set_rhs")
    n = tapes["fmg"][-1]
    x0 = state(s, cap, n)
    s.op("fmg", 0, 1 if first else 0)
    x1 = state(s, cap, n)
    y = forward(tapes["fmg1" if first else "fmg"], x0)
    phi = slice(4 * cap * SLOT, 5 * cap * SLOT)
    tmp = slice(5 * cap * SLOT, 6 * cap * SLOT)
    assert rel(y[phi], x1[phi]) < 1e-12
    assert rel(y[tmp], x1[tmp]) < 1e-12


def test_transport_phases_reproduce_the_oracle(mesh):
    s, cfg, cap, tapes = mesh
    n = tapes["copy"][-1]
    x0 = state(s, cap, n)
    s.op("copy_cc", 0, 2)
    s.op("copy_cc", 1, 3)
    assert rel(forward(tapes["copy"], x0), state(s, cap, n)) == 0
    dt = s.get_max_dt()
    s.op("fluxes_koren", dt)
    x0 = state(s, cap, n)
    s.op("consistent_fluxes")
    assert rel(forward(tapes["cons"], x0), state(s, cap, n)) < 1e-14
    s.op("update_solution", dt)
    x0 = state(s, cap, n)
    s.op("restrict_tree", 0)
    s.op("restrict_tree", 1)
    assert rel(forward(tapes["rstr"], x0), state(s, cap, n)) < 1e-14
    x0 = state(s, cap, n)
    s.op("set_rhs")
    assert rel(forward(tapes["rhs"], x0), state(s, cap, n)) < 1e-14
    x0 = state(s, cap, n)
    s.op("average_dens")
    assert rel(forward(tapes["avg"], x0), state(s, cap, n)) < 1e-15


def test_field_phases_reproduce_the_oracle(mesh):
    s, cfg, cap, tapes = mesh
    n = tapes["faces"][-1]
    x0 = state(s, cap, n)
    s.op("fld_from_pot")
    x1 = state(s, cap, n)
    faces = slice(NVC * cap * SLOT, n - 1)
    assert rel(forward(tapes["faces"], x0)[faces], x1[faces]) < 1e-14
    # the ghost cells of |E| are a function of the interior cells
    assert rel(forward(tapes["gcfld"], x1), x1) < 1e-14


@pytest.mark.parametrize("seg", list(SEG))
def test_transposed_phases_pass_the_dot_product_test(mesh, seg):
    s, cfg, cap, tapes = mesh
    pr, rd, rs, rt, ts, tc, n = tapes[seg]
    rng = np.random.default_rng(7)
    # each phase alone, to rounding
    for p in range(len(pr) - 1):
        r0, r1 = pr[p], pr[p + 1]
        one = (np.array([0, r1 - r0]), rd[r0:r1], rs[r0:r1], rt[r0:r1 + 1] - rt[r0],
               ts[rt[r0]:rt[r1]], tc[rt[r0]:rt[r1]], n)
        x, y = rng.standard_normal(n), rng.standard_normal(n)
        a, b = forward(one, x) @ y, x @ transpose(one, y)
        assert abs(a - b) <= 1e-12 * max(abs(a), 1.0), (seg, p)
    # the whole operation: hundreds of phases compose, and on random inputs
    # rounding grows through them (the first-call FMG reaches ~1e-8 in FP64
    # and ~1e-12 when the same test runs in 80-bit precision); a transposition
    # error shows at the per-phase test above and at the forward comparisons
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    a, b = forward(tapes[seg], x) @ y, x @ transpose(tapes[seg], y)
    assert abs(a - b) <= 1e-6 * abs(a)
