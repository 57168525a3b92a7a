"""CPU emulation of the device path's plan-based multigrid phases.

The device runs each phase as a flat, race-free parallel loop over the
(box, cell) items of one level, deriving every index from one record per box
(BoxRec, written by the host once per topology: build_plans in
a5_streamer_b200/csrc/a5g.cu, exported here through a5g_debug_plans, which
needs no GPU). This module replays the same phases with NumPy -- every phase
computes all of its outputs from the state before the phase, which is exactly
what the race-free parallel loop does -- in the same arithmetic order, so
that the plans and the phase schedule can be checked against the CPU oracle
without a GPU."""
from __future__ import annotations

import ctypes

import numpy as np

from a5_streamer_b200 import _lib

SLOT = 100
MAXLEV = 40
NBR_RB, NBR_PHYS = -1, -2
CF_LEAF, CF_PARENT = 1, 2
UC_EPS0 = 8.8541878176e-12
UC_ELEM_CHARGE = 1.6022e-19

BOXREC = np.dtype([("base", "i4"), ("pbase", "i4"), ("nb", "i4", 4), ("pnb", "i4", 4),
                   ("ch", "i4", 4), ("o0", "i4"), ("o1", "i4"), ("gi0", "i4"), ("flags", "i4"),
                   ("r0", "f8"), ("dr", "f8"), ("pad", "i4", 2)])
assert BOXREC.itemsize == 96


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Plans:
    def __init__(self, meta, geom, levels, min_lvl, max_lvl, dr_base):
        fn = _lib.lib().a5g_debug_plans
        counts, ids = [], []
        for lvl in range(min_lvl, max_lvl + 1):
            a, b, c = levels[lvl]
            counts += [len(a), len(b), len(c)]
            ids += list(a) + list(b) + list(c)
        counts = np.asarray(counts, dtype=np.int32)
        ids = np.asarray(ids, dtype=np.int32)
        meta = np.ascontiguousarray(meta, dtype=np.int32)
        geom = np.ascontiguousarray(geom, dtype=np.float64)
        args = [meta.shape[0] - 1, min_lvl, max_lvl, _ip(meta), _dp(geom), _ip(counts), _ip(ids),
                dr_base]
        sizes = np.zeros(2, dtype=np.int32)
        _lib.check(fn(*args, _ip(sizes), None, None, None, None, None))
        nlev = max_lvl - min_lvl + 1
        self.boxes = np.zeros(max(int(sizes[0]), 1), dtype=BOXREC)
        self.pbx = np.zeros(max(int(sizes[1]), 1), dtype=np.int32)
        offs = np.zeros(2 * (MAXLEV + 1), dtype=np.int32)
        self.lv_dr = np.zeros(nlev)
        self.lv_nc = np.zeros(nlev, dtype=np.int32)
        _lib.check(fn(*args, None, _ip(offs), self.boxes.ctypes.data_as(ctypes.c_void_p),
                      _ip(self.pbx), _dp(self.lv_dr), _ip(self.lv_nc)))
        self.bx_off, self.pb_off = offs[:MAXLEV + 1], offs[MAXLEV + 1:]
        self.min_lvl, self.max_lvl, self.nlev = min_lvl, max_lvl, nlev


class Emulator:
    """State: flat arrays (max_id+1) * SLOT per cell variable."""

    def __init__(self, plans: Plans, cc, coord, applied_voltage, n_cycle_base):
        self.P = plans
        self.cc = [np.array(x, dtype=np.float64).reshape(-1) for x in cc]
        self.cyl = coord == 1
        self.V = applied_voltage
        self.ncb = n_cycle_base

    def lvl(self, lvl):
        P = self.P
        li = lvl - P.min_lvl
        nc = int(P.lv_nc[li])
        return li, nc, nc + 2, P.boxes[P.bx_off[li]:P.bx_off[li + 1]], P.lv_dr[li]

    # ghosts ----------------------------------------------------------------
    def phi_ghost(self, phi, B, nc, ncg, side, k):
        """Vectorized over items: B records, side and k arrays."""
        dim, low = side >> 1, (side & 1) == 0
        nbb = B["nb"][np.arange(len(B)), side]
        out = np.empty(len(B))
        nbr = nbb > 0
        src = np.where(dim == 0, np.where(low, nc, 1) + ncg * k, k + ncg * np.where(low, nc, 1))
        out[nbr] = phi[nbb[nbr] + src[nbr]]
        ix = np.where(low, 1, nc)
        own = B["base"] + np.where(dim == 0, ix + ncg * k, k + ncg * ix)
        rb = nbb == NBR_RB
        if rb.any():
            di = np.where(low, 1, -1)
            dk = -1 + 2 * (k & 1)
            ig = ix - di
            o0, o1, pb = B["o0"], B["o1"], B["pbase"]
            pc = np.where(dim == 0, pb + (o0 + ((ig + 1) >> 1)) + ncg * (o1 + ((k + 1) >> 1)),
                          pb + (o0 + ((k + 1) >> 1)) + ncg * (o1 + ((ig + 1) >> 1)))
            a = np.where(dim == 0, own + di, own + dk)
            b = np.where(dim == 0, own + ncg * dk, own + ncg * di)
            out[rb] = (0.5 * phi[pc[rb]] + phi[own[rb]]) - 0.25 * (phi[a[rb]] + phi[b[rb]])
        ph = nbb == NBR_PHYS
        v = phi[own]
        out[ph & (side < 2)] = v[ph & (side < 2)]
        out[ph & (side == 2)] = -v[ph & (side == 2)]
        out[ph & (side == 3)] = 2 * self.V - v[ph & (side == 3)]
        return out

    def phi_ghost_flat(self, phi, B, nc, ncg, side, k):
        """The device's phi_ghost_flat: phi_ghost with the refinement-boundary
        source read from the parent's same-level neighbour (pnb) instead of
        the parent's ghost cell."""
        out = self.phi_ghost(phi, B, nc, ncg, side, k)
        dim, low = side >> 1, (side & 1) == 0
        rb = B["nb"][np.arange(len(B)), side] == NBR_RB
        if rb.any():
            ix = np.where(low, 1, nc)
            own = B["base"] + np.where(dim == 0, ix + ncg * k, k + ncg * ix)
            di = np.where(low, 1, -1)
            dk = -1 + 2 * (k & 1)
            xc = np.where(low, nc, 1)
            h2 = (k + 1) >> 1
            pn = B["pnb"][np.arange(len(B)), side]
            pc = pn + np.where(dim == 0, xc + ncg * (B["o1"] + h2), (B["o0"] + h2) + ncg * xc)
            a = np.where(dim == 0, own + di, own + dk)
            b = np.where(dim == 0, own + ncg * dk, own + ncg * di)
            out[rb] = (0.5 * phi[pc[rb]] + phi[own[rb]]) - 0.25 * (phi[a[rb]] + phi[b[rb]])
        return out

    def nbrs(self, phi, B, nc, ncg, i, j, g):
        vals = []
        for side, inner, k, off in ((0, i > 1, j, -1), (1, i < nc, j, 1), (2, j > 1, i, -ncg),
                                    (3, j < nc, i, ncg)):
            v = np.empty(len(g))
            v[inner] = phi[g[inner] + off]
            gh = ~inner
            if gh.any():
                v[gh] = self.phi_ghost(phi, B[gh], nc, ncg, np.full(gh.sum(), side), k[gh])
            vals.append(v)
        return vals

    def lap(self, phi, B, nc, ncg, i, j, inv):
        g = B["base"] + i + ncg * j
        lx, hx, ly, hy = self.nbrs(phi, B, nc, ncg, i, j, g)
        v = phi[g]
        if self.cyl:
            gi = (B["gi0"] + i).astype(np.float64)
            den = gi - 0.5
            rf1, rf2 = (gi - 1) / den, gi / den
            return (rf1 * lx + rf2 * hx + ly + hy - 4 * v) * inv
        return inv * (lx + hx + ly + hy - 4 * v)

    # item enumerations -------------------------------------------------------
    @staticmethod
    def cells(boxes, nc):
        nb = len(boxes)
        t = np.tile(np.arange(nc * nc), nb)
        B = np.repeat(boxes, nc * nc)
        return B, t % nc + 1, t // nc + 1

    @staticmethod
    def ghosts(boxes, nc):
        nb = len(boxes)
        r = np.tile(np.arange(4 * nc), nb)
        B = np.repeat(boxes, 4 * nc)
        return B, r // nc, r % nc + 1

    @staticmethod
    def ghost_dst(B, nc, ncg, side, k):
        gx = np.where(side & 1, nc + 1, 0)
        return B["base"] + np.where((side >> 1) == 0, gx + ncg * k, k + ncg * gx)

    # phases ------------------------------------------------------------------
    def sweep(self, lvl, it, mem=False):
        li, nc, ncg, boxes, dr = self.lvl(lvl)
        B, i, j = self.cells(boxes, nc)
        sel = ((i + j) & 1) == (it & 1)
        B, i, j = B[sel], i[sel], j[sel]
        phi, rhs = self.cc[4], self.cc[6]
        g = B["base"] + i + ncg * j
        if mem:
            lx, hx, ly, hy = phi[g - 1], phi[g + 1], phi[g - ncg], phi[g + ncg]
        else:
            lx, hx, ly, hy = self.nbrs(phi, B, nc, ncg, i, j, g)
        r = rhs[g]
        dx2 = dr * dr
        if self.cyl:
            gi = (B["gi0"] + i).astype(np.float64)
            den = gi - 0.5
            rf1, rf2 = (gi - 1) / den, gi / den
            new = 0.25 * (rf1 * lx + rf2 * hx + hy + ly - dx2 * r)
        else:
            new = 0.25 * (hx + lx + hy + ly - dx2 * r)
        phi[g] = new

    def fill_values(self, lvl):
        li, nc, ncg, boxes, dr = self.lvl(lvl)
        B, side, k = self.ghosts(boxes, nc)
        v = self.phi_ghost(self.cc[4], B, nc, ncg, side, k)
        return self.ghost_dst(B, nc, ncg, side, k), v, (B["flags"] & CF_PARENT) != 0

    def fill(self, lvl):
        d, v, _ = self.fill_values(lvl)
        self.cc[4][d] = v

    def fr_phase(self, lvl, fill, leaf_rhs, store_res):
        li, nc, ncg, boxes, dr = self.lvl(lvl)
        pncg = int(self.P.lv_nc[li - 1]) + 2
        phi, tmp, rhs, e, pi = self.cc[4], self.cc[5], self.cc[6], self.cc[0], self.cc[1]
        hn = nc // 2
        t = np.tile(np.arange(hn * hn), len(boxes))
        B = np.repeat(boxes, hn * hn)
        ii, jj = t % hn + 1, t // hn + 1
        inv = 1 / (dr * dr)
        fac = UC_ELEM_CHARGE / UC_EPS0
        if fill:
            fd, fv, _ = self.fill_values(lvl)
        leaf = ((B["flags"] & CF_LEAF) != 0) & leaf_rhs
        rs, ps, writes = [], [], []
        for q in range(4):
            i, j = 2 * ii - 1 + (q & 1), 2 * jj - 1 + (q >> 1)
            g = B["base"] + i + ncg * j
            rh = rhs[g].copy()
            rh[leaf] = fac * (e[g[leaf]] - pi[g[leaf]])
            res = rh - self.lap(phi, B, nc, ncg, i, j, inv)
            writes.append((g, rh, res))
            rs.append(res)
            ps.append(phi[g].copy())
        for g, rh, res in writes:
            rhs[g[leaf]] = rh[leaf]
            if store_res:
                tmp[g] = res
        d = B["pbase"] + (B["o0"] + ii) + pncg * (B["o1"] + jj)
        tmp[d] = 0.25 * (rs[0] + rs[1] + rs[2] + rs[3])
        phi[d] = 0.25 * (ps[0] + ps[1] + ps[2] + ps[3])
        if fill:
            phi[fd] = fv

    def fc_phase(self, lvl, copy_tmp):
        li, nc, ncg, boxes, dr = self.lvl(lvl)
        P = self.P
        pboxes = P.boxes[P.pbx[P.pb_off[li]:P.pb_off[li + 1]]]
        phi, tmp, rhs = self.cc[4], self.cc[5], self.cc[6]
        fd, fv, fpar = self.fill_values(lvl)
        if len(pboxes):
            B, i, j = self.cells(pboxes, nc)
            g = B["base"] + i + ncg * j
            a = self.lap(phi, B, nc, ncg, i, j, 1 / (dr * dr))
            newr, newt = a + tmp[g], phi[g].copy()
            rhs[g] = newr
            if copy_tmp:
                tmp[g] = newt
        phi[fd] = fv
        if copy_tmp:
            tmp[fd[fpar]] = fv[fpar]

    def correct(self, lvl, copy, corr):
        li, nc, ncg, boxes, dr = self.lvl(lvl)
        phi, tmp = self.cc[4], self.cc[5]
        B, i, j = self.cells(boxes, nc)
        g = B["base"] + i + ncg * j
        v = phi[g].copy()
        if corr:
            pncg = int(self.P.lv_nc[li - 1]) + 2
            i1 = B["o0"] + ((i + 1) >> 1)
            i2 = i1 + 1 - 2 * (i & 1)
            j1 = B["o1"] + ((j + 1) >> 1)
            j2 = j1 + 1 - 2 * (j & 1)
            p1 = B["pbase"] + i1 + pncg * j1
            p2 = B["pbase"] + i2 + pncg * j1
            p3 = B["pbase"] + i1 + pncg * j2
            newp = v + 0.5 * (phi[p1] - tmp[p1]) + 0.25 * ((phi[p2] - tmp[p2]) + (phi[p3] - tmp[p3]))
        if copy:
            Bg, side, k = self.ghosts(boxes, nc)
            d = self.ghost_dst(Bg, nc, ncg, side, k)
            gv = phi[d].copy()
            tmp[g] = v
            tmp[d] = gv
        if corr:
            phi[g] = newp

    def init_level(self, lvl, leaf_rhs):
        li, nc, ncg, boxes, dr = self.lvl(lvl)
        pncg = int(self.P.lv_nc[li - 1]) + 2
        rhs, phi, e, pi = self.cc[6], self.cc[4], self.cc[0], self.cc[1]
        hn = nc // 2
        t = np.tile(np.arange(hn * hn), len(boxes))
        B = np.repeat(boxes, hn * hn)
        ii, jj = t % hn + 1, t // hn + 1
        fac = UC_ELEM_CHARGE / UC_EPS0
        leaf = ((B["flags"] & CF_LEAF) != 0) & leaf_rhs
        rs = []
        for q in range(4):
            g = B["base"] + (2 * ii - 1 + (q & 1)) + ncg * (2 * jj - 1 + (q >> 1))
            rh = rhs[g].copy()
            rh[leaf] = fac * (e[g[leaf]] - pi[g[leaf]])
            rhs[g[leaf]] = rh[leaf]
            rs.append(rh)
        rhs[B["pbase"] + (B["o0"] + ii) + pncg * (B["o1"] + jj)] = 0.25 * (rs[0] + rs[1] + rs[2] + rs[3])
        for b in boxes:
            phi[b["base"]:b["base"] + ncg * ncg] = 0.0

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
