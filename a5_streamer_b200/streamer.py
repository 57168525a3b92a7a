"""Python mirror of the reference's streamer program and Afivo tree calls.

:class:`Tree` wraps the host quadtree (include/a5t.h: a$D_init,
a$D_set_base, a$D_adjust_refinement). :class:`Simulation` wraps the driver
(src/streamer_2d.f90 / src/streamer_cyl.f90 main program): ``init`` is the
initial refinement loop, ``advance`` one main-loop block (get_max_dt,
num_steps_amr time steps, regrid), ``run`` the loop to an end time. All box
data stay on the GPU; ``device`` gives the :class:`DeviceRun` view for
per-operation calls.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List

import numpy as np

from . import _lib
from ._lib import call, lib
from .config import TD_COLUMNS, StreamerConfig
from .device import DeviceRun, make_params


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Tree:
    """Host quadtree topology; ``handle`` may be borrowed from a Simulation."""

    def __init__(self, box_size=8, lvls_max=30, dr_base=1.0, r_base=(0.0, 0.0), coord=0,
                 handle=None):
        self._owned = handle is None
        if handle is None:
            h = ctypes.c_void_p()
            rb = np.asarray(r_base, dtype=np.float64)
            call("a5t_create", box_size, lvls_max, dr_base, _dp(rb), coord, ctypes.byref(h))
            handle = h
        self.h = handle

    def close(self):
        if self._owned and self.h is not None and self.h.value:
            lib().a5t_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_base(self, ix_list: np.ndarray, nb_list: np.ndarray):
        ix = np.ascontiguousarray(ix_list, dtype=np.int32)
        nb = np.ascontiguousarray(nb_list, dtype=np.int32)
        call("a5t_set_base", self.h, ix.shape[0], _ip(ix), _ip(nb))

    def adjust_refinement(self, flags: np.ndarray):
        f = np.ascontiguousarray(flags, dtype=np.int32)
        assert f.shape[0] >= self.max_id + 1
        a, r = ctypes.c_int(0), ctypes.c_int(0)
        call("a5t_adjust_refinement", self.h, _ip(f), ctypes.byref(a), ctypes.byref(r))
        return a.value, r.value

    @property
    def max_id(self) -> int:
        return lib().a5t_max_id(self.h)

    @property
    def min_lvl(self) -> int:
        return lib().a5t_min_lvl(self.h)

    @property
    def max_lvl(self) -> int:
        return lib().a5t_max_lvl(self.h)

    def export(self):
        n = lib().a5t_n_level_ids(self.h)
        meta = np.zeros((self.max_id + 1, 16), dtype=np.int32)
        geom = np.zeros((self.max_id + 1, 4))
        nlev = self.max_lvl - self.min_lvl + 1
        counts = np.zeros((nlev, 3), dtype=np.int32)
        ids = np.zeros(max(n, 1), dtype=np.int32)
        lib().a5t_export(self.h, _ip(meta), _dp(geom), _ip(counts), _ip(ids))
        levels, k = {}, 0
        for li in range(nlev):
            a, b, c = counts[li]
            levels[self.min_lvl + li] = (ids[k:k + a].copy(), ids[k + a:k + a + b].copy(),
                                         ids[k + a + b:k + a + b + c].copy())
            k += a + b + c
        return meta, geom, levels

    def new_boxes(self) -> Dict[int, List[int]]:
        nlev = self.max_lvl - self.min_lvl + 1
        counts = np.zeros(nlev, dtype=np.int32)
        tot = lib().a5t_new_boxes(self.h, None, None)
        ids = np.zeros(max(tot, 1), dtype=np.int32)
        lib().a5t_new_boxes(self.h, _ip(counts), _ip(ids))
        out, k = {}, 0
        for li in range(nlev):
            out[self.min_lvl + li] = ids[k:k + counts[li]].tolist()
            k += counts[li]
        return out


def base_grid(n_base):
    """ix_list / nb_list of a rectangular base grid with physical boundaries."""
    nx, ny = n_base
    ix = np.zeros((nx * ny, 2), dtype=np.int32)
    nb = np.zeros((nx * ny, 4), dtype=np.int32)
    for j in range(ny):
        for i in range(nx):
            k = i + nx * j
            ix[k] = (i + 1, j + 1)
            nb[k] = (k if i > 0 else -1, k + 2 if i < nx - 1 else -1,
                     k + 1 - nx if j > 0 else -1, k + 1 + nx if j < ny - 1 else -1)
    return ix, nb


class Simulation:
    """One streamer run on the GPU (host tree + device data)."""

    def __init__(self, cfg: StreamerConfig):
        cfg.validate()
        self.cfg = cfg
        sc = _lib.SimConfig()
        sc.dev = make_params(cfg)
        sc.n_base[0], sc.n_base[1] = cfg.n_base
        sc.bg_dens = cfg.bg_dens
        sc.n_seeds = len(cfg.seeds)
        for n, s in enumerate(cfg.seeds):
            sc.seed_dens[n] = s.dens
            sc.seed_falloff[n] = s.falloff
        sc.num_steps_amr = cfg.num_steps_amr
        sc.lkptbl_size = cfg.lkptbl_size
        sc.lkptbl_max_fld = cfg.lkptbl_max_fld
        kind, a, b = cfg.photoi_table
        sc.photoi_tbl_kind = 0 if kind == "air" else 1
        sc.photoi_tbl_a, sc.photoi_tbl_b = a, b
        sc.photoi_max_dist = cfg.photoi_max_dist
        self._keep = []
        for c, name in enumerate(TD_COLUMNS):
            xs = np.ascontiguousarray(cfg.td[name][0], dtype=np.float64)
            ys = np.ascontiguousarray(cfg.td[name][1], dtype=np.float64)
            self._keep += [xs, ys]
            sc.td_n[c] = len(xs)
            sc.td_x[c] = _dp(xs)
            sc.td_y[c] = _dp(ys)
        self._sc = sc
        h = ctypes.c_void_p()
        call("a5s_create", ctypes.byref(sc), ctypes.byref(h))
        self.h = h
        ctx = ctypes.c_void_p()
        call("a5s_ctx", self.h, ctypes.byref(ctx))
        th = ctypes.c_void_p()
        call("a5s_tree", self.h, ctypes.byref(th))
        self.tree = Tree(handle=th)
        self.device = DeviceRun.__new__(DeviceRun)
        self.device.cfg = cfg
        self.device.nc = cfg.box_size
        self.device.h = None  # borrowed context: never destroyed through this view
        self.device._borrowed = ctx
        self._refresh_view()

    def _refresh_view(self):
        d = self.device
        d.h = self.device._borrowed
        d.max_id = self.tree.max_id
        d.min_lvl = self.tree.min_lvl
        d.max_lvl = self.tree.max_lvl
        d.close = lambda: None

    def close(self):
        if self.h is not None and self.h.value:
            lib().a5s_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self) -> int:
        n = ctypes.c_int(0)
        call("a5s_init", self.h, ctypes.byref(n))
        self._refresh_view()
        return n.value

    def advance(self, regrid: bool = True) -> float:
        dt = ctypes.c_double(0)
        call("a5s_advance", self.h, 1 if regrid else 0, ctypes.byref(dt))
        self._refresh_view()
        return dt.value

    def run(self, t_end: float | None = None, max_blocks: int = 1 << 30) -> int:
        nb = ctypes.c_int(0)
        call("a5s_run", self.h, self.cfg.end_time if t_end is None else t_end, max_blocks,
             ctypes.byref(nb))
        self._refresh_view()
        return nb.value

    @property
    def time(self) -> float:
        t = ctypes.c_double(0)
        call("a5s_time", self.h, ctypes.byref(t))
        return t.value

    def table(self):
        n = ctypes.c_int(0)
        xm, inv = ctypes.c_double(0), ctypes.c_double(0)
        call("a5s_table", self.h, None, ctypes.byref(xm), ctypes.byref(inv), ctypes.byref(n))
        rc = np.zeros(4 * n.value)
        call("a5s_table", self.h, _dp(rc), None, None, None)
        return rc.reshape(4, n.value).T.copy(), xm.value, inv.value

    # -- checkpoint / resume (include/a5t.h a5s_checkpoint_*) ---------------
    def checkpoint(self) -> bytes:
        """The run's whole state (time, generator, tree, every cell and face
        variable) as bytes; ``restore`` on a run of the same configuration
        continues from it exactly."""
        n = ctypes.c_size_t(0)
        call("a5s_checkpoint_size", self.h, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value)
        w = ctypes.c_size_t(0)
        call("a5s_checkpoint_save", self.h, buf, n.value, ctypes.byref(w))
        return buf.raw[:w.value]

    def restore(self, data: bytes) -> None:
        call("a5s_checkpoint_load", self.h, data, len(data))
        self._refresh_view()

    def save(self, path: str) -> None:
        with open(path, "wb") as fh:
            fh.write(self.checkpoint())

    def load(self, path: str) -> None:
        with open(path, "rb") as fh:
            self.restore(fh.read())


def run_batch(sims, t_end, use_graph: bool = True, n_threads: int = 8, groups: int = 1,
              max_blocks: int = 1 << 30):
    """Run several simulations to their end times as one device-driven batch
    (include/a5t.h a5s_batch_run): per main-loop block one launch per kernel
    for all runs, replayed from a CUDA graph when ``use_graph``, regrids on
    the host in ``n_threads`` threads; with ``groups`` > 1 the runs are dealt
    to that many batches whose regrids overlap the others' device work. Each
    run ends in the state
    ``Simulation.run(t_end[k])`` gives it. Returns (blocks, device ms of the
    blocks, host ms of the regrids, leaf-cell updates over all runs)."""
    n = len(sims)
    if np.isscalar(t_end):
        t_end = [t_end] * n
    arr = (ctypes.c_void_p * n)(*[s.h.value for s in sims])
    te = np.ascontiguousarray(t_end, dtype=np.float64)
    nb = ctypes.c_int(0)
    g_ms, h_ms, cu = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
    call("a5s_batch_run", arr, n, _dp(te), 1 if use_graph else 0, int(n_threads), int(groups),
         int(max_blocks),
         ctypes.byref(nb), ctypes.byref(g_ms), ctypes.byref(h_ms), ctypes.byref(cu))
    for s in sims:
        s._refresh_view()
    return nb.value, g_ms.value, h_ms.value, cu.value
