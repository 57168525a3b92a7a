"""Gradients of a streamer-head observable with respect to the transport
parameters and the applied field (the differentiation addition).

The differentiated program P(p) runs on a fixed mesh with a fixed step-size
schedule:

1. ``set_init_cond`` on every box (the seed densities, phi = 0;
   src/streamer_2d.f90:218-248);
2. ``compute_fld`` with no guess, the first FMG call (src/streamer_2d.f90:307-343);
3. ``n_steps`` full time steps at the step sizes ``dts`` (one iteration of the
   n loop of src/streamer_2d.f90:93-128 each), no regrid;
4. J = the head height: over the leaf cells next to the line x = x0 (both
   sides; in the 8 mm case the symmetry line, a cell face), the mean of the
   cell heights weighted by dy * exp((|E| - max |E|) / T).

The softmax temperature T is a field. A length tau = 0.05 mm becomes
T = kappa tau^2 / 2, where kappa = -d^2|E|/dz^2 at the profile's maximum in
the nominal end state. For a parabolic peak the weights then fall off as
exp(-(z - z_max)^2 / tau^2). kappa is measured once on the nominal run and
then kept fixed, because it is part of the observable's definition.

The parameters p = (mobility, diffusion, alpha prefactor A, alpha exponent B,
E_bg) enter through the rows of the transport table (mu, D constant;
alpha = A exp(-B/|E|); eta = 0) and through the applied voltage
V = -L_z E_bg. The device adjoint (include/a5a.h) returns dJ/d(table rows)
and dJ/dV. :func:`param_tangents` maps both to dJ/dp.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence, Tuple

import numpy as np

from . import _lib, config
from ._lib import call

PARAM_NAMES = ("mobility", "diffusion", "alpha_a", "alpha_b", "applied_fld")


@dataclass
class HeadProblem:
    """The differentiated program: the 8 mm Cartesian case without
    photoionization, 200 steps, checkpoints every 20 steps."""
    n_steps: int = 200
    checkpoint_every: int = 20
    x0: float = 4e-3          # the line x = 4 mm
    tau: float = 0.05e-3      # smoothing length of the head observable

    @staticmethod
    def config():
        return config.cartesian_8mm()

    @staticmethod
    def nominal() -> np.ndarray:
        """p0 = (mu, D, A, B, E_bg) of the 8 mm case."""
        return np.array([0.03, 0.1, 4.3e5, 1.4e7, 2.5e6])


def table_rows(p: Sequence[float], n_rows: int = 200, x_max: float = 3e7) -> np.ndarray:
    """Table rows (n_rows x 4: mu, D, alpha, eta) of the synthetic transport
    data at parameters p, sampled at the table nodes as the nominal
    configuration is (config.synthetic_transport)."""
    td = config.synthetic_transport(n_rows, x_max, mobility=p[0], diffusion=p[1],
                                    alpha_a=p[2], alpha_b=p[3], eta_a=0.0)
    return np.array([td[name][1] for name in config.TD_COLUMNS]).T.copy()


def param_tangents(p: Sequence[float], domain_len_z: float, n_rows: int = 200,
                   x_max: float = 3e7) -> Tuple[np.ndarray, np.ndarray]:
    """Derivatives of the table rows (5 x n_rows x 4) and of the applied
    voltage (5,) with respect to each parameter."""
    xs = np.array(config.table_nodes(n_rows, x_max))
    d = np.zeros((5, n_rows, 4))
    dV = np.zeros(5)
    d[0, :, 0] = 1.0
    d[1, :, 1] = 1.0
    pos = xs > 0
    e = np.zeros(n_rows)
    e[pos] = np.exp(-p[3] / xs[pos])
    d[2, :, 2] = e                       # d alpha / dA
    d[3, pos, 2] = -p[2] / xs[pos] * e[pos]  # d alpha / dB
    dV[4] = -domain_len_z                # V = -L_z E_bg
    return d, dV


def chain_to_params(dJ_table: np.ndarray, dJ_dV: float, p: Sequence[float],
                    domain_len_z: float) -> np.ndarray:
    """dJ/dp from dJ/d(table rows) (n_rows x 4) and dJ/dV."""
    d, dV = param_tangents(p, domain_len_z, dJ_table.shape[0])
    return np.einsum("krc,rc->k", d, dJ_table) + dV * dJ_dV


def head_temperature(profile: np.ndarray, tau: float) -> float:
    """T = kappa tau^2 / 2 from a head profile (rows: y, dy, |E|), with kappa
    the curvature of |E| along y at its maximum. Both columns next to the
    line share heights in a symmetric mesh; equal heights are averaged first."""
    y = np.round(profile[:, 0], 12)
    ys = np.unique(y)
    E = np.array([profile[y == v, 2].mean() for v in ys])
    k = int(np.argmax(E))
    if k == 0 or k == len(ys) - 1:
        raise ValueError("the |E| maximum lies at the end of the profile")
    ym, y0, yp = ys[k - 1:k + 2]
    Em, E0, Ep = E[k - 1:k + 2]
    kappa = -2.0 * ((Ep - E0) / (yp - y0) - (E0 - Em) / (y0 - ym)) / (yp - ym)
    if not kappa > 0:
        raise ValueError("no curvature at the |E| maximum")
    return 0.5 * kappa * tau * tau


def head_profile(meta: np.ndarray, geom: np.ndarray, levels, E: np.ndarray, x0: float,
                 nc: int = 8) -> np.ndarray:
    """(y, dy, |E|) of the leaf cells next to the line x = x0 (either side),
    levels in order, leaves in list order, cells by height: the profile the
    observable is taken over. E is the |E| variable in slot layout."""
    out = []
    for lvl in sorted(levels):
        for id_ in levels[lvl][1]:
            r0, r1, dr = geom[id_, 0], geom[id_, 1], geom[id_, 3]
            n = meta[id_, 14]
            tol = 1e-9 * dr
            if abs(r0 + n * dr - x0) <= tol:
                i = n
            elif abs(r0 - x0) <= tol:
                i = 1
            else:
                continue
            for j in range(1, n + 1):
                out.append((r1 + (j - 0.5) * dr, dr, E[id_, i + (n + 2) * j]))
    return np.array(out).reshape(-1, 3)


AdjParams = _lib.AdjParams


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def debug_tape(meta, geom, levels, capacity: int, n_cycle_base: int, seg: int):
    """The transposed phases of one operation (a5a_debug_tape), as arrays
    (phase_row, row_d, row_self, row_term, term_s, term_c, vector length)."""
    meta = np.ascontiguousarray(meta, dtype=np.int32)
    geom = np.ascontiguousarray(geom, dtype=np.float64)
    lo, hi = min(levels), max(levels)
    counts, ids = [], []
    for lvl in range(lo, hi + 1):
        a, b, c = levels[lvl]
        counts += [len(a), len(b), len(c)]
        ids += list(a) + list(b) + list(c)
    counts = np.asarray(counts, dtype=np.int32)
    ids = np.asarray(ids if ids else [0], dtype=np.int32)
    sizes = (ctypes.c_longlong * 4)()
    args = (meta.shape[0] - 1, lo, hi, _ip(meta), _dp(geom), _ip(counts), _ip(ids), capacity,
            n_cycle_base, seg, sizes)
    call("a5a_debug_tape", *args, None, None, None, None, None, None)
    n_p, n_r, n_t, n_x = (int(v) for v in sizes)
    pr = np.zeros(n_p + 1, dtype=np.int32)
    rd = np.zeros(max(n_r, 1), dtype=np.uint32)
    rs = np.zeros(max(n_r, 1))
    rt = np.zeros(n_r + 1, dtype=np.int32)
    ts = np.zeros(max(n_t, 1), dtype=np.uint32)
    tc = np.zeros(max(n_t, 1))
    u = ctypes.POINTER(ctypes.c_uint)
    call("a5a_debug_tape", *args, _ip(pr), rd.ctypes.data_as(u), _dp(rs), _ip(rt),
         ts.ctypes.data_as(u), _dp(tc))
    return pr, rd[:n_r], rs[:n_r], rt, ts[:n_t], tc[:n_t], n_x


class HeadAdjoint:
    """Device adjoint (include/a5a.h) of the head observable on the fixed mesh
    of an initialised :class:`streamer.Simulation`.

    ``schedule`` runs the nominal program once to record the step sizes (one
    get_max_dt per block of num_steps_amr steps, as the main loop takes
    them) and the softmax temperature; ``value`` and ``gradient`` evaluate P
    at parameters p, setting the run's table and applied field first."""

    def __init__(self, sim, problem: HeadProblem | None = None):
        self.sim = sim
        self.prob = problem or HeadProblem()
        self.cfg = sim.cfg
        self.ctx = sim.device._borrowed
        self.h = None
        self.dts = None
        self.temperature = None
        tab, self.x_min, self.inv_dx = sim.table()
        self.n_rows = tab.shape[0]

    def set_params(self, p) -> None:
        rows = table_rows(p, self.n_rows, self.cfg.lkptbl_max_fld)
        flat = np.ascontiguousarray(rows.T.reshape(-1))
        call("a5g_set_table", self.ctx, self.n_rows, 4, self.x_min, self.inv_dx, _dp(flat))
        call("a5g_set_applied_field", self.ctx, float(p[4]))

    def schedule(self, p=None):
        """Record dts and T on the nominal trajectory; returns (dts, T)."""
        p = self.prob.nominal() if p is None else p
        self.set_params(p)
        call("a5s_set_init_cond", self.sim.h)
        dev = self.sim.device
        dev.compute_fld(True)
        dts = []
        while len(dts) < self.prob.n_steps:
            dt = ctypes.c_double(0)
            call("a5g_get_max_dt", self.ctx, ctypes.byref(dt))
            for _ in range(self.cfg.num_steps_amr):
                call("a5g_step", self.ctx, dt.value)
                dts.append(dt.value)
        self.dts = np.array(dts[:self.prob.n_steps])
        meta, geom, levels = self.sim.tree.export()
        prof = head_profile(meta, geom, levels, dev.cc(5), self.prob.x0, self.cfg.box_size)
        self.temperature = head_temperature(prof, self.prob.tau)
        return self.dts, self.temperature

    def bind(self, dts=None, temperature=None):
        """Create the device adjoint; the run is put in the initial state."""
        if dts is not None:
            self.dts = np.ascontiguousarray(dts, dtype=np.float64)
        if temperature is not None:
            self.temperature = float(temperature)
        if self.dts is None or self.temperature is None:
            raise ValueError("call schedule() or pass dts and temperature")
        self.close()
        call("a5s_set_init_cond", self.sim.h)
        ap = AdjParams(len(self.dts), self.prob.checkpoint_every, self.prob.x0, self.temperature)
        h = ctypes.c_void_p()
        d = np.ascontiguousarray(self.dts, dtype=np.float64)
        call("a5a_create", self.ctx, ctypes.byref(ap), _dp(d), ctypes.byref(h))
        self.h = h
        return self

    def close(self):
        if self.h is not None and self.h.value:
            _lib.lib().a5a_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def value(self, p) -> float:
        self.set_params(p)
        J = ctypes.c_double(0)
        call("a5a_forward", self.h, ctypes.byref(J))
        return J.value

    def gradient_raw(self, p):
        """(J, dJ/d(table rows) n_rows x 4, dJ/dV) at parameters p."""
        self.set_params(p)
        J = ctypes.c_double(0)
        dV = ctypes.c_double(0)
        g = np.zeros(4 * self.n_rows)
        call("a5a_gradient", self.h, ctypes.byref(J), _dp(g), ctypes.byref(dV))
        return J.value, g.reshape(4, self.n_rows).T.copy(), dV.value

    def gradient(self, p):
        """(J, dJ/dp) at parameters p = (mu, D, A, B, E_bg)."""
        J, gt, gv = self.gradient_raw(p)
        return J, chain_to_params(gt, gv, p, self.cfg.domain_len_z)
