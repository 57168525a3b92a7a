"""The 3D octree form of the device path (include/a5g3.h) from Python.

One :class:`Run3` is one run on a uniformly refined octree, resident on the
current CUDA device. The octree is built by the library with the reference's
box ids (a3_set_base then refinement level by level); cell and face data use
the reference's per-id slot layouts, so arrays exchange directly with other
implementations of the same tree.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .config import TD_COLUMNS, StreamerConfig, table_nodes

_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_IP)


def make_params3(cfg: StreamerConfig) -> _lib.Params3:
    cfg.validate()
    if cfg.dim != 3:
        raise ValueError("Run3 takes a 3D configuration")
    p = _lib.Params3()
    p.box_size = cfg.box_size
    for d in range(3):
        p.n_base[d] = cfg.n_base[d]
    p.uniform_lvl = cfg.uniform_lvl
    p.n_cycle_base = cfg.n_cycle_base
    p.use_drt = 1 if cfg.use_drt else 0
    p.dr_base = cfg.dr_base
    p.domain_len_z = cfg.domain_len_z
    p.applied_fld = cfg.applied_fld
    p.dt_max = cfg.dt_max
    return p


def transport_table(cfg: StreamerConfig):
    """The lookup table of LT_create / LT_set_col (fosito/m_lookup_table.f90:
    46-72, 200-221): n_rows x 4 column-major, x_min, inv_dx."""
    n = cfg.lkptbl_size
    xs = np.array(table_nodes(n, cfg.lkptbl_max_fld))
    cols = []
    for name in TD_COLUMNS:
        x, y = (np.asarray(v, dtype=np.float64) for v in cfg.td[name])
        cols.append(_lin_interp_list(x, y, xs))
    rc = np.ascontiguousarray(np.concatenate(cols))
    return rc, 0.0, (n - 1) / (cfg.lkptbl_max_fld - 0.0), n


def _lin_interp_list(xl: np.ndarray, yl: np.ndarray, xs: np.ndarray) -> np.ndarray:
    # LT_lin_interp_list (fosito/m_lookup_table.f90:200-221) with
    # find_index_adaptive (fosito/m_find_index.f90:26-67), per node
    out = np.empty(len(xs))
    n = len(xl)
    for q, x in enumerate(xs):
        if x <= xl[0]:
            out[q] = yl[0]
        elif x >= xl[n - 1]:
            out[q] = yl[n - 1]
        else:
            ix = int(np.searchsorted(xl, x, side="left")) + 1  # smallest ix with x <= xl[ix-1]
            temp = (x - xl[ix - 2]) / (xl[ix - 1] - xl[ix - 2])
            out[q] = (1 - temp) * yl[ix - 2] + temp * yl[ix - 1]
    return out


class Run3:
    """One 3D run on a uniformly refined octree, on the current CUDA device."""

    def __init__(self, cfg: StreamerConfig, table=None):
        self.cfg = cfg
        self._p = make_params3(cfg)
        h = ctypes.c_void_p()
        _lib.call3("a5g3_create", ctypes.byref(self._p), ctypes.byref(h))
        self.h = h
        mid, lo, hi = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        nl = ctypes.c_longlong()
        _lib.call3("a5g3_info", self.h, ctypes.byref(mid), ctypes.byref(lo), ctypes.byref(hi),
                   ctypes.byref(nl))
        self.max_id, self.min_lvl, self.max_lvl, self.n_leaf_cells = mid.value, lo.value, hi.value, nl.value
        self.nc = cfg.box_size
        rc, x_min, inv_dx, n_rows = table if table is not None else transport_table(cfg)
        rc = np.ascontiguousarray(rc, dtype=np.float64)
        _lib.call3("a5g3_set_table", self.h, n_rows, 4, x_min, inv_dx, _dp(rc))

    def close(self):
        if self.h:
            _lib.lib().a5g3_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- tree ----------------------------------------------------------------
    def meta(self) -> np.ndarray:
        m = np.zeros((self.max_id + 1, 24), dtype=np.int32)
        _lib.call3("a5g3_export_meta", self.h, _ip(m))
        return m

    def levels(self):
        nlev = self.max_lvl - self.min_lvl + 1
        counts = np.zeros((nlev, 3), dtype=np.int32)
        cap = 3 * (self.max_id + 1)
        ids = np.zeros(cap, dtype=np.int32)
        n = ctypes.c_int()
        _lib.call3("a5g3_export_levels", self.h, _ip(counts), _ip(ids), cap, ctypes.byref(n))
        out, k = {}, 0
        for li in range(nlev):
            n_ids, n_lv, n_pa = counts[li]
            a = ids[k:k + n_ids].copy(); k += n_ids
            b = ids[k:k + n_lv].copy(); k += n_lv
            c = ids[k:k + n_pa].copy(); k += n_pa
            out[self.min_lvl + li] = (a, b, c)
        return out

    # --- data ----------------------------------------------------------------
    def set_init_cond(self):
        cfg = self.cfg
        n = len(cfg.seeds)
        r0 = np.array([s.r0 for s in cfg.seeds], dtype=np.float64).reshape(-1)
        r1 = np.array([s.r1 for s in cfg.seeds], dtype=np.float64).reshape(-1)
        dens = np.array([s.dens for s in cfg.seeds], dtype=np.float64)
        width = np.array([s.width for s in cfg.seeds], dtype=np.float64)
        fall = np.array([s.falloff for s in cfg.seeds], dtype=np.int32)
        _lib.call3("a5g3_set_init_cond", self.h, cfg.bg_dens, n, _dp(r0), _dp(r1), _dp(dens), _dp(width),
                   _ip(fall))

    def cc(self, iv: int) -> np.ndarray:
        out = np.zeros((self.max_id + 1, (self.nc + 2) ** 3))
        _lib.call3("a5g3_download_cc", self.h, iv, _dp(out))
        return out

    def set_cc(self, iv: int, data: np.ndarray):
        data = np.ascontiguousarray(data, dtype=np.float64)
        if data.size != (self.max_id + 1) * (self.nc + 2) ** 3:
            raise ValueError("cell data has the wrong size")
        _lib.call3("a5g3_upload_cc", self.h, iv, _dp(data))

    def fc(self, dimf: int, f: int) -> np.ndarray:
        out = np.zeros((self.max_id + 1, (self.nc + 1) * self.nc * self.nc))
        _lib.call3("a5g3_download_fc", self.h, dimf, f, _dp(out))
        return out

    def set_fc(self, dimf: int, f: int, data: np.ndarray):
        data = np.ascontiguousarray(data, dtype=np.float64)
        if data.size != (self.max_id + 1) * (self.nc + 1) * self.nc * self.nc:
            raise ValueError("face data has the wrong size")
        _lib.call3("a5g3_upload_fc", self.h, dimf, f, _dp(data))

    # --- operations ------------------------------------------------------------
    def op(self, name: str, *args):
        _lib.call3("a5g3_" + name, self.h, *args)

    def compute_fld(self, no_guess: bool = False):
        self.op("compute_fld", 1 if no_guess else 0)

    def init(self):
        """Initial conditions on the uniform mesh and the first field solve
        (src/streamer_3d.f90:55-61 on the final mesh, phi from 0)."""
        self.set_init_cond()
        self.compute_fld(True)

    def dt_reductions(self) -> np.ndarray:
        out = np.zeros(3)
        _lib.call3("a5g3_dt_reductions", self.h, _dp(out))
        return out

    def get_max_dt(self) -> float:
        out = ctypes.c_double()
        _lib.call3("a5g3_get_max_dt", self.h, ctypes.byref(out))
        return out.value

    def tree_max_cc(self, iv: int) -> float:
        out = ctypes.c_double()
        _lib.call3("a5g3_tree_max_cc", self.h, iv, ctypes.byref(out))
        return out.value

    def tree_min_cc(self, iv: int) -> float:
        out = ctypes.c_double()
        _lib.call3("a5g3_tree_min_cc", self.h, iv, ctypes.byref(out))
        return out.value

    def step(self, dt: float):
        _lib.call3("a5g3_step", self.h, dt)

    def set_precision(self, mixed: bool, schedule=None):
        """FP64 (the reference's arithmetic) or the mixed form (include/a5g3.h
        a5g3_set_precision); schedule: (fmg, n_cycle_down, n_cycle_up,
        n_cycle_base, n_corr) of the FP32 correction solve, None for the
        reference's."""
        sp = None
        if schedule is not None:
            sp = ctypes.byref(_lib.MGSchedule(*[int(v) for v in schedule]))
        _lib.call3("a5g3_set_precision", self.h, _lib.A5G_MIXED if mixed else _lib.A5G_FP64, sp)

    def sync(self):
        _lib.call3("a5g3_sync", self.h)

    def stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        _lib.call3("a5g3_stream", self.h, ctypes.byref(s))
        return s.value or 0

    def bytes_per_step(self) -> float:
        """Compulsory-traffic model of one full step on this tree (the FP64
        words each phase must read and write once; see metrics.bytes_per_step
        for the 2D form): per leaf cell of the 3D step about 3.4 kB."""
        from . import metrics
        return metrics.bytes_per_step_3d(self)


def leaf_cells(level: int, n_base=(1, 1, 1), nc: int = 8) -> int:
    return int(math.prod(n_base)) * (8 ** (level - 1)) * nc ** 3
