"""CPU emulation of the device path's plan-based multigrid and field phases.

The device runs each phase as a flat, race-free parallel loop over a plan
(cell table, ghost recipes, restriction records) that the host builds once
per topology (build_plans in a5_streamer_b200/csrc/a5g.cu, exported here
through a5g_debug_plans, which needs no GPU). This module replays the same
phases with NumPy -- every phase computes all of its outputs from the state
before the phase, which is exactly what the race-free parallel loop does --
in the same arithmetic order, so that the plans and the phase schedule can
be checked against the CPU oracle without a GPU."""
from __future__ import annotations

import ctypes

import numpy as np

from a5_streamer_b200 import _lib

SLOT = 100
MAXLEV = 40
NB_MASK = 0x0FFFFFFF
GK_COPY, GK_NEG, GK_APPLIED, GK_RB, GK_INTERP = range(5)
GK_PARENT = 0x100
CF_LEAF = 1
UC_EPS0 = 8.8541878176e-12
UC_ELEM_CHARGE = 1.6022e-19


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Plans:
    def __init__(self, meta, geom, levels, min_lvl, max_lvl, dr_base, coord):
        L = _lib.lib()
        fn = L.a5g_debug_plans
        fn.restype = ctypes.c_int
        counts, ids = [], []
        for lvl in range(min_lvl, max_lvl + 1):
            a, b, c = levels[lvl]
            counts += [len(a), len(b), len(c)]
            ids += list(a) + list(b) + list(c)
        counts = np.asarray(counts, dtype=np.int32)
        ids = np.asarray(ids, dtype=np.int32)
        meta = np.ascontiguousarray(meta, dtype=np.int32)
        geom = np.ascontiguousarray(geom, dtype=np.float64)
        max_id = meta.shape[0] - 1
        sizes = np.zeros(6, dtype=np.int32)
        args = [ctypes.c_int(max_id), ctypes.c_int(min_lvl), ctypes.c_int(max_lvl), _ip(meta),
                _dp(geom), _ip(counts), _ip(ids), ctypes.c_double(dr_base), ctypes.c_int(coord)]
        null = [None] * 11
        _lib.check(fn(*args, _ip(sizes), *null))
        nc, ng, nd, nr, nf, npc = (int(x) for x in sizes)
        self.offs = np.zeros(7 * (MAXLEV + 1), dtype=np.int32)
        self.cells = np.zeros((max(nc, 1), 12), dtype=np.int32)
        self.gphi = np.zeros((max(ng, 1), 6), dtype=np.int32)
        self.gden = np.zeros((max(nd, 1), 6), dtype=np.int32)
        self.rst_i = np.zeros((max(nr, 1), 2), dtype=np.int32)
        self.rst_rfac = np.zeros(max(nr, 1))
        self.fr = np.zeros((max(nf, 1), 8), dtype=np.int32)
        self.pcells = np.zeros(max(npc, 1), dtype=np.int32)
        nlev = max_lvl - min_lvl + 1
        self.lv_dr = np.zeros(nlev)
        self.lv_nc = np.zeros(nlev, dtype=np.int32)
        _lib.check(fn(*args, None, _ip(self.offs), _ip(self.cells), _ip(self.gphi), _ip(self.gden),
                      _ip(self.rst_i), _dp(self.rst_rfac), _ip(self.fr), _ip(self.pcells),
                      _dp(self.lv_dr), _ip(self.lv_nc)))
        o = self.offs.reshape(7, MAXLEV + 1)
        self.cell_off, self.cell_split, self.gphi_off, self.gden_off = o[0], o[1], o[2], o[3]
        self.rst_off, self.fr_off, self.pcell_off = o[4], o[5], o[6]
        self.min_lvl, self.max_lvl, self.nlev = min_lvl, max_lvl, nlev
        self.levels = levels


class Emulator:
    """State: flat arrays (max_id+1) * SLOT per cell variable, faces likewise."""

    def __init__(self, plans: Plans, cc, fx, fy, coord, applied_voltage, n_cycle_base):
        self.P = plans
        self.cc = [np.array(x, dtype=np.float64).reshape(-1) for x in cc]
        self.fx = [np.array(x, dtype=np.float64).reshape(-1) for x in fx]
        self.fy = [np.array(x, dtype=np.float64).reshape(-1) for x in fy]
        self.cyl = coord == 1
        self.V = applied_voltage
        self.ncb = n_cycle_base

    # helpers ---------------------------------------------------------------
    def recipe(self, x, recs):
        kind = recs[:, 1] & 0xFF
        s = recs[:, 2:6]
        out = np.empty(len(recs))
        m = kind == GK_COPY
        out[m] = x[s[m, 0]]
        m = kind == GK_NEG
        out[m] = -x[s[m, 0]]
        m = kind == GK_APPLIED
        out[m] = 2 * self.V - x[s[m, 0]]
        m = kind == GK_RB
        out[m] = 0.5 * x[s[m, 0]] + x[s[m, 1]] - 0.25 * (x[s[m, 2]] + x[s[m, 3]])
        return out

    def nbv(self, x, codes, gl):
        kind = (codes.astype(np.int64) & 0xFFFFFFFF) >> 28
        idx = codes & NB_MASK
        out = np.empty(len(codes))
        m = kind == 0
        out[m] = x[idx[m]]
        m = kind == 1
        out[m] = -x[idx[m]]
        m = kind == 2
        out[m] = 2 * self.V - x[idx[m]]
        m = kind == 3
        if m.any():
            out[m] = self.recipe(x, gl[idx[m]])
        return out

    def lap(self, phi, c, gl, inv_dr_sq):
        lx, hx = self.nbv(phi, c[:, 1], gl), self.nbv(phi, c[:, 2], gl)
        ly, hy = self.nbv(phi, c[:, 3], gl), self.nbv(phi, c[:, 4], gl)
        v = phi[c[:, 0]]
        if self.cyl:
            gi = c[:, 8].astype(np.float64)
            den = gi - 0.5
            rf1, rf2 = (gi - 1) / den, gi / den
            return (rf1 * lx + rf2 * hx + ly + hy - 4 * v) * inv_dr_sq
        return inv_dr_sq * (lx + hx + ly + hy - 4 * v)

    def li(self, lvl):
        return lvl - self.P.min_lvl

    def gl(self, li):
        P = self.P
        return P.gphi[P.gphi_off[li]:P.gphi_off[li + 1]]

    # phases ------------------------------------------------------------------
    def sweep(self, lvl, it, mem=False):
        P, li = self.P, self.li(lvl)
        phi, rhs = self.cc[4], self.cc[6]
        a, b = (P.cell_split[li], P.cell_off[li + 1]) if it & 1 else (P.cell_off[li], P.cell_split[li])
        c = P.cells[a:b]
        if len(c) == 0:
            return
        gl = self.gl(li)
        dr = P.lv_dr[li]
        dx2 = dr * dr
        ncg = P.lv_nc[li] + 2
        g = c[:, 0]
        if mem:
            lx, hx, ly, hy = phi[g - 1], phi[g + 1], phi[g - ncg], phi[g + ncg]
        else:
            lx, hx = self.nbv(phi, c[:, 1], gl), self.nbv(phi, c[:, 2], gl)
            ly, hy = self.nbv(phi, c[:, 3], gl), self.nbv(phi, c[:, 4], gl)
        r = rhs[g]
        if self.cyl:
            gi = c[:, 8].astype(np.float64)
            den = gi - 0.5
            rf1, rf2 = (gi - 1) / den, gi / den
            new = 0.25 * (rf1 * lx + rf2 * hx + hy + ly - dx2 * r)
        else:
            new = 0.25 * (hx + lx + hy + ly - dx2 * r)
        phi[g] = new

    def fill_values(self, li):
        gl = self.gl(li)
        return gl, self.recipe(self.cc[4], gl)

    def fill(self, lvl):
        gl, v = self.fill_values(self.li(lvl))
        self.cc[4][gl[:, 0]] = v

    def fr_phase(self, lvl, fill, leaf_rhs, store_res):
        P, li = self.P, self.li(lvl)
        phi, tmp, rhs, e, pi = self.cc[4], self.cc[5], self.cc[6], self.cc[0], self.cc[1]
        recs = P.fr[P.fr_off[li]:P.fr_off[li + 1]]
        gl = self.gl(li)
        dr = P.lv_dr[li]
        inv = 1 / (dr * dr)
        fac = UC_ELEM_CHARGE / UC_EPS0
        if fill:
            gfl, gv = self.fill_values(li)
        rs, ps = [], []
        rhs_w, tmp_w = [], []
        for q in range(4):
            c = P.cells[recs[:, 1 + q]]
            g = c[:, 0]
            rh = rhs[g].copy()
            if leaf_rhs:
                m = (c[:, 9] & CF_LEAF) != 0
                rh[m] = fac * (e[g[m]] - pi[g[m]])
                rhs_w.append((g[m], rh[m]))
            res = rh - self.lap(phi, c, gl, inv)
            if store_res:
                tmp_w.append((g, res))
            rs.append(res)
            ps.append(phi[g].copy())
        for g, v in rhs_w:
            rhs[g] = v
        for g, v in tmp_w:
            tmp[g] = v
        tmp[recs[:, 0]] = 0.25 * (rs[0] + rs[1] + rs[2] + rs[3])
        phi[recs[:, 0]] = 0.25 * (ps[0] + ps[1] + ps[2] + ps[3])
        if fill:
            phi[gfl[:, 0]] = gv

    def fc_phase(self, lvl, copy_tmp):
        P, li = self.P, self.li(lvl)
        phi, tmp, rhs = self.cc[4], self.cc[5], self.cc[6]
        c = P.cells[P.pcells[P.pcell_off[li]:P.pcell_off[li + 1]]]
        gl = self.gl(li)
        dr = P.lv_dr[li]
        inv = 1 / (dr * dr)
        gfl, gv = self.fill_values(li)
        if len(c):
            g = c[:, 0]
            a = self.lap(phi, c, gl, inv)
            newr = a + tmp[g]
            newt = phi[g].copy()
            rhs[g] = newr
            if copy_tmp:
                tmp[g] = newt
        phi[gfl[:, 0]] = gv
        if copy_tmp:
            m = (gfl[:, 1] & GK_PARENT) != 0
            tmp[gfl[m, 0]] = gv[m]

    def correct(self, lvl, copy, corr):
        P, li = self.P, self.li(lvl)
        phi, tmp = self.cc[4], self.cc[5]
        c = P.cells[P.cell_off[li]:P.cell_off[li + 1]]
        g = c[:, 0]
        v = phi[g].copy()
        if corr:
            c1 = phi[c[:, 5]] - tmp[c[:, 5]]
            c2x = phi[c[:, 6]] - tmp[c[:, 6]]
            c2y = phi[c[:, 7]] - tmp[c[:, 7]]
            newp = v + 0.5 * c1 + 0.25 * (c2x + c2y)
        if copy:
            gl = self.gl(li)
            gv = phi[gl[:, 0]].copy()
            tmp[g] = v
            tmp[gl[:, 0]] = gv
        if corr:
            phi[g] = newp

    def init_level(self, lvl, leaf_rhs):
        P, li = self.P, self.li(lvl)
        rhs, phi, e, pi = self.cc[6], self.cc[4], self.cc[0], self.cc[1]
        recs = P.fr[P.fr_off[li]:P.fr_off[li + 1]]
        fac = UC_ELEM_CHARGE / UC_EPS0
        rs = []
        for q in range(4):
            c = P.cells[recs[:, 1 + q]]
            g = c[:, 0]
            rh = rhs[g].copy()
            if leaf_rhs:
                m = (c[:, 9] & CF_LEAF) != 0
                rh[m] = fac * (e[g[m]] - pi[g[m]])
                rhs[g[m]] = rh[m]
            rs.append(rh)
        rhs[recs[:, 0]] = 0.25 * (rs[0] + rs[1] + rs[2] + rs[3])
        ids = P.levels[lvl][0]
        per = (P.lv_nc[li] + 2) ** 2
        for i in ids:
            phi[i * SLOT:i * SLOT + per] = 0.0

    def vcycle(self, max_lvl, stale_base):
        mn = self.P.min_lvl
        for lvl in range(max_lvl, mn, -1):
            for it in range(1, 5):
                self.sweep(lvl, it)
            self.fr_phase(lvl, True, False, False)
            self.fc_phase(lvl - 1, True)
        for it in range(1, 2 * self.ncb + 1):
            self.sweep(mn, it, stale_base and it == 1)
        self.fill(mn)
        for lvl in range(mn + 1, max_lvl + 1):
            self.correct(lvl, False, True)
            for it in range(1, 5):
                self.sweep(lvl, it)
            self.fill(lvl)

    def fmg(self, first_call, leaf_rhs):
        mn, mx = self.P.min_lvl, self.P.max_lvl
        if first_call:
            for lvl in range(mx, mn, -1):
                self.init_level(lvl, leaf_rhs)
        else:
            for lvl in range(mx, mn, -1):
                self.fr_phase(lvl, lvl == mx, leaf_rhs, True)
                self.fc_phase(lvl - 1, False)
        for lvl in range(mn, mx + 1):
            self.correct(lvl, True, lvl > mn)
            self.vcycle(lvl, first_call and lvl == mn)
