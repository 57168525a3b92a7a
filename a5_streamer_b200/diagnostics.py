"""Streamer diagnostics of the axisymmetric program, computed on the host
from the arrays a run downloads (or any arrays in the device layout):

- ``streamer_properties``: the 39 properties of get_streamer_properties
  (src/streamer_cyl.f90:682-828): background field, maximum axial and radial
  field and their locations, the radius, the head potential and density, the
  potential drop ahead of the head, and the radial / axial extent of the
  region above field thresholds 4..14 MV/m;
- ``axis_data``: get_cc_axis (:905-956), the cell column next to the axis
  box by box from z = 0 up: z, n_e, n_i, the axial field and the axial
  electron flux (face averages).

The tree helpers restate afivo/src/m_aX_utils.f90: a$D_get_loc (:244-281,
descent to the finest box below lvls_max that contains the point,
a$D_cc_ix with ``ceiling``), a$D_reduction_loc (:499-555, leaves level by
level in list order; a box replaces the running result only when the
reduction changes it, so ties keep the first location) and
a$D_r_cc / a$D_r_loc (cell centres).

One property restates a quirk of the reference. The "mobility" that
get_streamer_properties uses for S = alpha * mu * E is read from the alpha
column (:708-709, :718-719).
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

C_MOB, C_DIF, C_ALPHA, C_ETA = range(4)


class TreeView:
    """Read-only view of a tree in the device layout (meta16, geom4, level
    lists) with the box accessors the diagnostics need."""

    def __init__(self, meta: np.ndarray, geom: np.ndarray, levels, lvls_max: int):
        self.meta, self.geom, self.levels, self.lvls_max = meta, geom, levels, lvls_max

    def nc(self, bid: int) -> int:
        return int(self.meta[bid, 14])

    def lvl(self, bid: int) -> int:
        return int(self.meta[bid, 1])

    def r_min(self, bid: int) -> Tuple[float, float]:
        return float(self.geom[bid, 0]), float(self.geom[bid, 1])

    def dr(self, bid: int) -> float:
        return float(self.geom[bid, 3])

    def children(self, bid: int) -> List[int]:
        return [int(c) for c in self.meta[bid, 6:10]]

    def leaves(self):
        for lvl in sorted(self.levels):
            for bid in self.levels[lvl][1]:
                yield int(bid)

    def r_cc(self, bid: int, i: int, j: int) -> Tuple[float, float]:
        r0, r1 = self.r_min(bid)
        dr = self.dr(bid)
        return r0 + (i - 0.5) * dr, r1 + (j - 0.5) * dr

    def get_loc(self, rr: Sequence[float]) -> Tuple[int, Tuple[int, int]]:
        """a$D_get_loc: (id, (i, j)) of the cell containing rr, id -1 outside."""
        bid = -1
        for b in self.levels.get(1, ([], [], []))[0]:
            r0, r1 = self.r_min(int(b))
            n, dr = self.nc(int(b)), self.dr(int(b))
            if rr[0] >= r0 and rr[1] >= r1 and rr[0] <= r0 + dr * n and rr[1] <= r1 + dr * n:
                bid = int(b)
                break
        if bid < 0:
            return -1, (-1, -1)
        while self.lvl(bid) < self.lvls_max and self.children(bid)[0] != 0:
            r0, r1 = self.r_min(bid)
            c0 = r0 + self.dr(bid) * (self.nc(bid) >> 1)
            c1 = r1 + self.dr(bid) * (self.nc(bid) >> 1)
            k = (1 if rr[0] > c0 else 0) + (2 if rr[1] > c1 else 0)
            bid = self.children(bid)[k]
        r0, r1 = self.r_min(bid)
        dr = self.dr(bid)
        return bid, (math.ceil((rr[0] - r0) / dr), math.ceil((rr[1] - r1) / dr))


def reduction_max_loc(tv: TreeView, box_fn, init: float):
    """a$D_reduction_loc with reduce_max, one thread: (value, (id, (i, j)))."""
    my_val, my_loc = init, (-1, (-1, -1))
    for bid in tv.leaves():
        tmp, ix = box_fn(bid)
        new = max(tmp, my_val)
        if abs(new - my_val) > 0:
            my_loc = (bid, ix)
            my_val = tmp
    new = max(my_val, init)
    if abs(new - init) > 0:
        return my_val, my_loc
    return init, (-1, (-1, -1))


def lt_col(table, col: int, x: float) -> float:
    """LT_get_col (fosito/m_lookup_table.f90:107-161) on a table
    (rows_cols, x_min, inv_dx) as returned by Simulation.table()."""
    rc, x_min, inv_dx = table
    n_rows = rc.shape[0]
    frac = (x - x_min) * inv_dx
    if -2.0e9 < frac < 2.0e9:
        ix = math.ceil(frac)
        fr = ix - frac
    else:
        ix, fr = (n_rows if frac > 0 else 0), 0.0
    if ix < 1:
        ix, fr = 1, 1.0
    elif ix >= n_rows:
        ix, fr = n_rows - 1, 0.0
    return fr * rc[ix - 1, col] + (1 - fr) * rc[ix, col]


def streamer_properties(tv: TreeView, cc: Dict[str, np.ndarray], fc: Dict[str, np.ndarray],
                        table, applied_fld: float, applied_voltage: float,
                        domain_len: float) -> Tuple[List[str], np.ndarray]:
    """get_streamer_properties (src/streamer_cyl.f90:682-828). cc: 'fld',
    'e', 'phi' cell variables; fc: 'fx_fld', 'fy_fld' face variables (one
    slot per box id, the device layout). Returns (names, values)."""
    fld, dens, phi = cc["fld"], cc["e"], cc["phi"]
    fx, fy = fc["fx_fld"], fc["fy_fld"]

    def fxv(bid, i, j):
        n = tv.nc(bid)
        return fx[bid, (i - 1) + (n + 1) * (j - 1)]

    def fyv(bid, i, j):
        n = tv.nc(bid)
        return fy[bid, (i - 1) + n * (j - 1)]

    def cell(v, bid, i, j):
        n = tv.nc(bid)
        return v[bid, i + (n + 2) * j]

    def maxfld(bid, radial):
        # maxloc over |f(lo) + f(hi)|, column-major (i fastest), first maximum
        n = tv.nc(bid)
        best, ix = -1.0, (1, 1)
        for j in range(1, n + 1):
            for i in range(1, n + 1):
                s = abs(fxv(bid, i, j) + fxv(bid, i + 1, j)) if radial else \
                    abs(fyv(bid, i, j) + fyv(bid, i, j + 1))
                if s > best:
                    best, ix = s, (i, j)
        i, j = ix
        v = 0.5 * abs(fxv(bid, i, j) + fxv(bid, i + 1, j)) if radial else \
            0.5 * abs(fyv(bid, i, j) + fyv(bid, i, j + 1))
        return v, ix

    def fld_max_pos(bid, thr, axis):
        n = tv.nc(bid)
        val, ix = 0.0, (-1, -1)
        for j in range(1, n + 1):
            for i in range(1, n + 1):
                if cell(fld, bid, i, j) > thr:
                    r = tv.r_cc(bid, i, j)
                    if r[axis] > val:
                        val, ix = r[axis], (i, j)
        return val, ix

    names, props = [], []

    def add(name, v):
        names.append(name)
        props.append(float(v))

    add("E_bg", applied_fld)
    ez_max, loc_ez = reduction_max_loc(tv, lambda b: maxfld(b, False), -1.0e99)
    add("Ez_max", ez_max)
    er_max, loc_er = reduction_max_loc(tv, lambda b: maxfld(b, True), -1.0e99)
    add("Er_max", er_max)
    rz = tv.r_cc(loc_er[0], *loc_er[1])
    add("Er_max(r)", rz[0])
    add("Er_max(z)", rz[1])
    z_head = rz[1]
    er_norm = cell(fld, loc_er[0], *loc_er[1])
    add("Er_max(E)", er_norm)
    for name, e in (("Ez_max", ez_max), ("Er_max", er_norm)):
        alpha = lt_col(table, C_ALPHA, e)
        mu = lt_col(table, C_ALPHA, e)  # the reference reads mu from the alpha column
        add(f"{name}(alpha)", alpha)
        add(f"{name}(S)", alpha * mu * e)
    bid, ix = tv.get_loc((0.0, rz[1]))
    add("n_e(head)", cell(dens, bid, *ix))
    phi_head = cell(phi, bid, *ix)
    add("dphi", phi_head - (rz[1] / domain_len) * applied_voltage)
    rz = tv.r_cc(loc_ez[0], *loc_ez[1])
    add("Ez_max(z)", rz[1])
    for dz, name in ((2.0e-3, "dphi(2mm)"), (4.0e-3, "dphi(4mm)")):
        b2, ix2 = tv.get_loc((0.0, rz[1] + dz))
        add(name, phi_head - cell(phi, b2, *ix2) if b2 > 0 else 0.0)
    for k in range(4, 16, 2):
        thr = k * 1e6
        v, loc = reduction_max_loc(tv, lambda b: fld_max_pos(b, thr, 0), 0.0)
        add(f"r_max({k}e6)", v)
        add(f"dphi_r({k}e6)", phi_head - cell(phi, loc[0], *loc[1]) if loc[0] > 0 else 0.0)
        v, loc = reduction_max_loc(tv, lambda b: fld_max_pos(b, thr, 1), 0.0)
        add(f"z_max({k}e6)", v - z_head)
        add(f"dphi_z({k}e6)", phi_head - cell(phi, loc[0], *loc[1]) if loc[0] > 0 else 0.0)
    return names, np.asarray(props)


def axis_data(tv: TreeView, cc_vars: Sequence[np.ndarray], fy_vars: Sequence[np.ndarray]) -> np.ndarray:
    """get_cc_axis (src/streamer_cyl.f90:905-956): rows z, the cell variables
    of the first cell column, then the face averages 0.5 (fy(1, j) +
    fy(1, j+1)) of the face variables, box by box from z = 0 up."""
    cols = []
    z = 0.0
    while True:
        bid, _ = tv.get_loc((0.0, z))
        if bid == -1:
            break
        n, dz = tv.nc(bid), tv.dr(bid)
        box_z = tv.r_min(bid)[1]
        j = np.arange(1, n + 1)
        rows = [box_z + (j - 0.5) * dz]
        for v in cc_vars:
            rows.append(np.asarray(v)[bid, 1 + (n + 2) * j])
        for f in fy_vars:
            f = np.asarray(f)
            rows.append(0.5 * (f[bid, 0 + n * (j - 1)] + f[bid, 0 + n * j]))
        cols.append(np.stack(rows))
        z = box_z + (n + 1) * dz
    return np.concatenate(cols, axis=1) if cols else np.zeros((1 + len(cc_vars) + len(fy_vars), 0))


def run_properties(sim):
    """streamer_properties and axis_data of a Simulation's current state (the
    output of write_streamer_properties, src/streamer_cyl.f90:647-680)."""
    cfg = sim.cfg
    meta, geom, levels = sim.tree.export()
    tv = TreeView(meta, geom, levels, cfg.lvls_max)
    d = sim.device
    cc = {"fld": d.cc(5), "e": d.cc(0), "phi": d.cc(4)}
    fc = {"fx_fld": d.fc(0, 1), "fy_fld": d.fc(1, 1)}
    names, props = streamer_properties(tv, cc, fc, sim.table(), cfg.applied_fld,
                                       cfg.applied_voltage, cfg.domain_len_z)
    axis = axis_data(tv, [d.cc(0), d.cc(1)], [d.fc(1, 1), d.fc(1, 0)])
    return dict(zip(names, props)), axis
