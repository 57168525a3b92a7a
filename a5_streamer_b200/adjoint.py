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
