"""Throughput accounting: tree census and the algorithmic-bytes model of one
full time step.

The model counts compulsory traffic: every phase of the step reads each
distinct input field once and writes each output once over the interior
cells, plus ghost traffic of g = 4D/nc words per variable per ghost fill.
Per full step (two forward-Euler stages, two field solves, the trapezoidal
average; src/streamer_2d.f90:93-128), in 8-byte words:

  T1 save old densities        4 N_all
  T2 fluxes + update (x2)      2 (3D + 7 + 2D/nc) N_leaf
  T3 restriction (x2)          2 * 2 (1 + 2^-D) N_{l>=2}
  T4 ghost fill n_e, n_i (x2)  2 * 2 g N_all
  T5 average                   6 N_all
  T6 space charge (x2)         2 * 3 N_leaf
  T7 FAS FMG (x2)              2 [ sum_l N_l ((L-l+1) V + F) + 5 sum_l P_l (L-l+1) ]
                               V = 2(n_down+n_up) 2.5 + 2(n_down+n_up) g + 3 + 2(1+2^-D) + 2 + 2 + g
                               F = 12 + 2g
  T8 field from potential (x2) 2 (D + 2 + g) N_all
  T9 step-size reductions      3 N_leaf

with N_l the cells of all boxes on level l, P_l the cells of parent boxes on
level l, L the finest level, N_all = sum over levels >= 1, N_leaf the leaf
cells. For a uniform 2D tree this is about 253 words (2 kB) per leaf cell.

With photoionization (src/streamer_cyl.f90:572-617, once per step) add

  T10 photon sources           8 N_leaf words + 16 bytes per photon

(production rate: read |E| and n_e, write the rate; the sum and the
creation pass read the rate; the photon count per cell is written and read;
the source term is written; per photon a 4-byte source cell written and
read and a 4-byte counter read and written).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Tuple

import numpy as np


@dataclass
class Census:
    dim: int
    nc: int
    min_lvl: int
    max_lvl: int
    cells: Dict[int, int]         # all boxes per level
    leaf_cells: Dict[int, int]
    parent_cells: Dict[int, int]

    @property
    def n_leaf(self) -> int:
        return sum(self.leaf_cells.values())

    @property
    def n_all(self) -> int:
        return sum(v for l, v in self.cells.items() if l >= 1)


def census(meta: np.ndarray, levels: Dict[int, Tuple[np.ndarray, np.ndarray, np.ndarray]],
           nc: int, dim: int = 2) -> Census:
    cells, leaf, par = {}, {}, {}
    for lvl, (ids, lv, pa) in levels.items():
        cnt = lambda xs: int(sum(int(meta[i, 14]) ** dim for i in xs))
        cells[lvl], leaf[lvl], par[lvl] = cnt(ids), cnt(lv), cnt(pa)
    return Census(dim, nc, min(levels), max(levels), cells, leaf, par)


def census3(meta24: np.ndarray, levels, nc: int) -> Census:
    """Census of a 3D octree from its 24-int meta rows (n_cell in column 20)."""
    cells, leaf, par = {}, {}, {}
    for lvl, (ids, lv, pa) in levels.items():
        cnt = lambda xs: int(sum(int(meta24[i, 20]) ** 3 for i in xs))
        cells[lvl], leaf[lvl], par[lvl] = cnt(ids), cnt(lv), cnt(pa)
    return Census(3, nc, min(levels), max(levels), cells, leaf, par)


def bytes_per_step_3d(run) -> float:
    """The model above with D = 3 (g = 1.5 words per variable per ghost fill at
    nc = 8) on a 3D run's tree (device3.Run3)."""
    return bytes_per_step(census3(run.meta(), run.levels(), run.nc))


def bytes_per_step(c: Census, n_down: int = 2, n_up: int = 2, word: int = 8,
                   photons: float = 0.0) -> float:
    """Algorithmic bytes of one full step; photons > 0 adds the photon
    sources of a step with photoionization and that many photons."""
    D, nc = c.dim, c.nc
    g = 4.0 * D / nc
    N_all, N_leaf = c.n_all, c.n_leaf
    N_ge2 = sum(v for l, v in c.cells.items() if l >= 2)
    t1 = 4 * N_all
    t2 = 2 * (3 * D + 7 + 2.0 * D / nc) * N_leaf
    t3 = 2 * 2 * (1 + 2.0 ** -D) * N_ge2
    t4 = 2 * 2 * g * N_all
    t5 = 6 * N_all
    t6 = 2 * 3 * N_leaf
    V = 2 * (n_down + n_up) * 2.5 + 2 * (n_down + n_up) * g + 3 + 2 * (1 + 2.0 ** -D) + 2 + 2 + g
    F = 12 + 2 * g
    L = c.max_lvl
    fmg = sum(n * ((L - l + 1) * V + F) for l, n in c.cells.items())
    fmg += 5 * sum(n * (L - l + 1) for l, n in c.parent_cells.items())
    t7 = 2 * fmg
    t8 = 2 * (D + 2 + g) * N_all
    t9 = 3 * N_leaf
    total = word * (t1 + t2 + t3 + t4 + t5 + t6 + t7 + t8 + t9)
    if photons > 0:
        total += word * 8 * N_leaf + 16.0 * photons
    return total


# ---------------------------------------------------------------------------
# Observables of the streamer head, used to state the error of the mixed
# form against the FP64 path.

def line_cells(meta: np.ndarray, geom: np.ndarray, levels, cfg):
    """Leaf cells along the symmetry line: the axis r = 0 of the cylindrical
    form (the first cell column of the boxes that touch it), or the line
    x = L/2 of the Cartesian form (the two cell columns beside it). Returns
    (box ids, cell indices into the (nc+2)^2 slot, z of the cell centres)."""
    ids, cells, zs = [], [], []
    x_line = 0.0 if cfg.coord == "cyl" else 0.5 * cfg.domain_len[0]
    for lvl, (_, leaves, _) in levels.items():
        for bid in leaves:
            n = int(meta[bid, 14])
            dr = geom[bid, 3]
            r0, r1 = geom[bid, 0], geom[bid, 1]
            for i in range(1, n + 1):
                xc = r0 + (i - 0.5) * dr
                if abs(xc - x_line) >= dr:
                    continue
                for j in range(1, n + 1):
                    ids.append(bid)
                    cells.append(i + (n + 2) * j)
                    zs.append(r1 + (j - 0.5) * dr)
    return np.asarray(ids), np.asarray(cells), np.asarray(zs)


def head_observables(fld: np.ndarray, meta, geom, levels, cfg):
    """(z of the maximum of |E| on the symmetry line, that maximum, the
    maximum of |E| over all leaf cells). fld: the |E| cell variable as
    downloaded, one (nc+2)^2 slot per box id."""
    ids, cells, zs = line_cells(meta, geom, levels, cfg)
    vals = fld[ids, cells]
    k = int(np.argmax(vals))
    emax = 0.0
    for lvl, (_, leaves, _) in levels.items():
        for bid in leaves:
            n = int(meta[bid, 14])
            blk = fld[bid, :(n + 2) ** 2].reshape(n + 2, n + 2)[1:n + 1, 1:n + 1]
            emax = max(emax, float(blk.max()))
    return float(zs[k]), float(vals[k]), emax
