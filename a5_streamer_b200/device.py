"""Device-resident run: Python mirror of the reference's Afivo/streamer call
surface over the C ABI (include/a5g.h).

Names follow the reference: ``tree_copy_cc`` (a$D_tree_copy_cc),
``fluxes_koren``, ``consistent_fluxes``, ``update_solution``,
``restrict_tree``, ``gc_tree``, ``average_dens``, ``compute_fld``,
``fas_fmg``, ``get_max_dt``, ``ref_flags`` (set_ref_flags over the tree) and
``prolong_to_new_boxes``. Errors raise :class:`A5GError` with the status code
the reference would have ``stop``-ped on.
"""
from __future__ import annotations

import ctypes
from typing import Dict, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import call, lib

I_ELEC, I_PION, I_ELEC_OLD, I_PION_OLD, I_PHI, I_FLD, I_RHS, I_PHO, I_EPS = range(9)
F_ELEC, F_FLD = 0, 1
N_VAR_CELL, N_VAR_FACE = 9, 2
RB_INTERP_LIM, RB_INTERP = 0, 1


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def make_params(cfg) -> _lib.Params:
    p = _lib.Params()
    p.box_size = cfg.box_size
    p.coord = 1 if cfg.coord == "cyl" else 0
    p.lvls_max = cfg.lvls_max
    p.dr_base = cfg.dr_base
    p.domain_len_z = cfg.domain_len_z
    p.applied_fld = cfg.applied_fld
    p.epsilon_diel = cfg.epsilon_diel
    p.dt_max = cfg.dt_max
    p.use_drt = 1 if cfg.use_drt else 0
    p.n_cycle_base = cfg.n_cycle_base
    p.ref_init_time = cfg.ref_init_time
    p.crv_refine = cfg.crv_refine
    p.n_seeds = len(cfg.seeds)
    for n, s in enumerate(cfg.seeds):
        for d in range(2):
            p.seed_r0[n][d] = s.r0[d]
            p.seed_r1[n][d] = s.r1[d]
        p.seed_width[n] = s.width
    p.photoi_enabled = 1 if cfg.photoi_enabled else 0
    p.photoi_num_photons = cfg.photoi_num_photons
    p.photoi_team = cfg.photoi_team
    p.photoi_coeff = cfg.photoi_coeff
    p.photoi_fac_dx = cfg.photoi_fac_dx
    for i in range(4):
        p.rng_seed[i] = cfg.rng_seed[i]
    p.uniform_lvl = cfg.uniform_lvl
    return p


def photon_table(cfg) -> Tuple[np.ndarray, float]:
    """PH_get_tbl_air-style absorption table of a configuration
    (src/m_photons.f90:25-93) built by the library's host code: 500
    distances at cumulative fractions (i-1)/499, and frac_in_tbl."""
    kind, a, b = cfg.photoi_table
    dist = np.zeros(500)
    frac, n = ctypes.c_double(0), ctypes.c_int(0)
    call("a5t_photon_table", 0 if kind == "air" else 1, a, b, cfg.photoi_max_dist, _dp(dist),
         ctypes.byref(frac), ctypes.byref(n))
    return dist[:n.value], frac.value


class DeviceRun:
    """One run (tree + box data) resident on the GPU."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.nc = cfg.box_size
        self._params = make_params(cfg)
        h = ctypes.c_void_p()
        call("a5g_create", ctypes.byref(self._params), ctypes.byref(h))
        self.h = h
        self.max_id = 0
        self.min_lvl = self.max_lvl = 0

    def close(self):
        if self.h is not None and self.h.value:
            lib().a5g_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # setup --------------------------------------------------------------------
    def set_table(self, rows_cols: np.ndarray, x_min: float, inv_dx: float):
        rc = np.asfortranarray(rows_cols, dtype=np.float64)
        n_rows, n_cols = rc.shape
        flat = np.ascontiguousarray(rc.T.reshape(-1))  # column-major
        call("a5g_set_table", self.h, n_rows, n_cols, x_min, inv_dx, _dp(flat))

    def upload_tree(self, meta: np.ndarray, geom: np.ndarray, min_lvl: int, max_lvl: int,
                    levels: Dict[int, Tuple[np.ndarray, np.ndarray, np.ndarray]]):
        meta = np.ascontiguousarray(meta, dtype=np.int32)
        geom = np.ascontiguousarray(geom, dtype=np.float64)
        counts, ids = [], []
        for lvl in range(min_lvl, max_lvl + 1):
            a, b, c = levels[lvl]
            counts += [len(a), len(b), len(c)]
            ids += list(a) + list(b) + list(c)
        counts = np.asarray(counts, dtype=np.int32)
        ids = np.asarray(ids if ids else [0], dtype=np.int32)
        max_id = meta.shape[0] - 1
        call("a5g_upload_tree", self.h, max_id, min_lvl, max_lvl, _ip(meta), _dp(geom),
             _ip(counts), _ip(ids))
        self.max_id, self.min_lvl, self.max_lvl = max_id, min_lvl, max_lvl

    # data ---------------------------------------------------------------------
    def cc(self, iv: int) -> np.ndarray:
        out = np.zeros((self.max_id + 1, (self.nc + 2) ** 2))
        call("a5g_download_cc", self.h, iv, _dp(out))
        return out

    def set_cc(self, iv: int, data: np.ndarray):
        data = np.ascontiguousarray(data, dtype=np.float64)
        assert data.shape == (self.max_id + 1, (self.nc + 2) ** 2)
        call("a5g_upload_cc", self.h, iv, _dp(data))

    def fc(self, dimf: int, f: int) -> np.ndarray:
        out = np.zeros((self.max_id + 1, (self.nc + 1) * self.nc))
        call("a5g_download_fc", self.h, dimf, f, _dp(out))
        return out

    def set_fc(self, dimf: int, f: int, data: np.ndarray):
        data = np.ascontiguousarray(data, dtype=np.float64)
        call("a5g_upload_fc", self.h, dimf, f, _dp(data))

    # box-loop operations ------------------------------------------------------
    def tree_copy_cc(self, iv_from: int, iv_to: int):
        call("a5g_tree_copy_cc", self.h, iv_from, iv_to)

    def fluxes_koren(self, dt: float):
        call("a5g_fluxes_koren", self.h, dt)

    def consistent_fluxes(self):
        call("a5g_consistent_fluxes", self.h)

    def update_solution(self, dt: float):
        call("a5g_update_solution", self.h, dt)

    def restrict_tree(self, iv: int):
        call("a5g_restrict_tree", self.h, iv)

    def gc_tree(self, iv: int, rb_kind: int = RB_INTERP_LIM):
        call("a5g_gc_tree", self.h, iv, rb_kind)

    def average_dens(self):
        call("a5g_average_dens", self.h)

    def compute_fld(self, no_guess: bool = False):
        call("a5g_compute_fld", self.h, 1 if no_guess else 0)

    def fas_fmg(self, set_residual: bool, first_call: bool):
        call("a5g_fas_fmg", self.h, 1 if set_residual else 0, 1 if first_call else 0)

    def fas_vcycle(self, max_lvl: int, set_residual: bool = False):
        """mg$D_fas_vcycle (afivo/src/m_aX_mg.f90:208-254)."""
        call("a5g_mg_fas_vcycle", self.h, int(max_lvl), 1 if set_residual else 0)

    def tree_max_cc(self, iv: int) -> float:
        """a$D_tree_max_cc: max over the leaves' interior cells."""
        out = ctypes.c_double()
        call("a5g_tree_max_cc", self.h, iv, ctypes.byref(out))
        return out.value

    def tree_min_cc(self, iv: int) -> float:
        """a$D_tree_min_cc: min over the leaves' interior cells."""
        out = ctypes.c_double()
        call("a5g_tree_min_cc", self.h, iv, ctypes.byref(out))
        return out.value

    def tree_sum_cc(self, iv: int, team: int = 1) -> float:
        """a$D_tree_sum_cc as an OpenMP team of `team` threads forms it."""
        out = ctypes.c_double()
        call("a5g_tree_sum_cc", self.h, iv, int(team), ctypes.byref(out))
        return out.value

    def fld_from_pot(self):
        call("a5g_fld_from_pot", self.h)

    def dt_reductions(self) -> np.ndarray:
        out = np.zeros(3)
        call("a5g_dt_reductions", self.h, _dp(out))
        return out

    def get_max_dt(self) -> float:
        out = ctypes.c_double(0)
        call("a5g_get_max_dt", self.h, ctypes.byref(out))
        return out.value

    def ref_flags(self, time: float) -> np.ndarray:
        out = np.zeros(self.max_id + 1, dtype=np.int32)
        call("a5g_ref_flags", self.h, time, _ip(out))
        return out

    def prolong_to_new_boxes(self, new_by_level: Dict[int, Sequence[int]]):
        counts = np.asarray([len(new_by_level.get(l, ())) for l in range(self.min_lvl, self.max_lvl + 1)],
                            dtype=np.int32)
        ids = [i for l in range(self.min_lvl, self.max_lvl + 1) for i in new_by_level.get(l, ())]
        ids = np.asarray(ids if ids else [0], dtype=np.int32)
        call("a5g_prolong_new", self.h, _ip(counts), _ip(ids))

    def step(self, dt: float):
        call("a5g_step", self.h, dt)

    def set_precision(self, mixed: bool, schedule=None):
        """Plain FP64 (the reference's arithmetic) or the mixed form: FP32
        fluxes, lookups and multigrid smoothing inside an FP64 defect
        correction. schedule: (fmg, n_cycle_down, n_cycle_up, n_cycle_base,
        n_corr) of the FP32 solve; None keeps the reference's schedule."""
        sp = None
        if schedule is not None:
            sp = ctypes.byref(_lib.MGSchedule(*[int(v) for v in schedule]))
        call("a5g_set_precision", self.h, _lib.A5G_MIXED if mixed else _lib.A5G_FP64, sp)

    def precision(self):
        """(mixed?, schedule tuple)"""
        p, s = ctypes.c_int(0), _lib.MGSchedule()
        call("a5g_get_precision", self.h, ctypes.byref(p), ctypes.byref(s))
        return p.value == _lib.A5G_MIXED, (s.fmg, s.n_cycle_down, s.n_cycle_up, s.n_cycle_base,
                                            s.n_corr)

    def set_photon_table(self, dist: np.ndarray, frac_in_tbl: float, x_min: float = 0.0,
                         inv_dx: float | None = None):
        d = np.ascontiguousarray(dist, dtype=np.float64)
        if inv_dx is None:
            inv_dx = (len(d) - 1) / 1.0
        call("a5g_set_photon_table", self.h, len(d), x_min, inv_dx, _dp(d), frac_in_tbl)

    def photoionization(self, dt: float | None):
        """set_photoionization (src/streamer_cyl.f90:572-593); dt None is the
        call before the time loop."""
        call("a5g_photoionization", self.h, 0.0 if dt is None else dt, 0 if dt is None else 1)

    def photon_stats(self) -> Tuple[int, float]:
        """(photons created by the last photoionization call, its fac)"""
        n, fac = ctypes.c_longlong(0), ctypes.c_double(0)
        call("a5g_photon_stats", self.h, ctypes.byref(n), ctypes.byref(fac))
        return n.value, fac.value

    def rng_state(self) -> np.ndarray:
        st = np.zeros(4, dtype=np.int32)
        call("a5g_get_rng", self.h, _ip(st))
        return st

    def set_rng_state(self, st) -> None:
        st = np.ascontiguousarray(st, dtype=np.int32)
        call("a5g_set_rng", self.h, _ip(st))

    def set_ctas(self, n_cta: int, wait_cycles: int = -1):
        """Grid mode: the run's phases on n_cta co-resident thread blocks
        (a5g_set_ctas); 1 is one block. wait_cycles bounds each barrier wait
        (< 0: the library's default)."""
        call("a5g_set_ctas", self.h, int(n_cta), int(wait_cycles))

    def set_level_set(self, lsf, bval):
        """Level-set boundaries of the field solve (a5g_set_level_set): per
        cell the level-set function and the boundary potential, downloaded
        layout; None, None removes them."""
        if lsf is None:
            call("a5g_set_level_set", self.h, None, None)
            return
        lsf = np.ascontiguousarray(lsf, dtype=np.float64)
        bval = np.ascontiguousarray(bval, dtype=np.float64)
        call("a5g_set_level_set", self.h, _dp(lsf), _dp(bval))

    def set_grid_local(self, cells: int):
        """Grid mode: levels of at most `cells` cells run on one block."""
        call("a5g_set_grid_local", self.h, int(cells))

    def ctas(self) -> Tuple[int, int]:
        """(blocks per launch of this run, most blocks the device can hold at once)"""
        n, m = ctypes.c_int(0), ctypes.c_int(0)
        call("a5g_get_ctas", self.h, ctypes.byref(n), ctypes.byref(m))
        return n.value, m.value

    def sync(self):
        call("a5g_sync", self.h)

    def stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        call("a5g_get_stream", self.h, ctypes.byref(s))
        return s.value or 0

    def n_leaf_cells(self) -> int:
        n = ctypes.c_longlong(0)
        call("a5g_n_leaf_cells", self.h, ctypes.byref(n))
        return n.value


def step_batch(runs: Sequence[DeviceRun], dts: Sequence[float]):
    n = len(runs)
    arr = (ctypes.c_void_p * n)(*[r.h.value for r in runs])
    d = np.ascontiguousarray(dts, dtype=np.float64)
    call("a5g_step_batch", arr, n, _dp(d))


def clone_state(sim, mixed: bool = False, schedule=None, cfg=None) -> DeviceRun:
    """A new device run holding a copy of ``sim``'s current tree, cell and face
    data, transport table, photon table and generator state (the state a
    reference run holds between two steps), in the given precision. cfg: a
    variant of the run's configuration (e.g. photoionization off)."""
    cfg = sim.cfg if cfg is None else cfg
    src = sim.device
    meta, geom, levels = sim.tree.export()
    rc, xm, inv = sim.table()
    r = DeviceRun(cfg)
    r.set_table(rc, xm, inv)
    if cfg.photoi_enabled:
        ph_dist, ph_frac = photon_table(cfg)
        r.set_photon_table(ph_dist, ph_frac)
        r.set_rng_state(src.rng_state())
    r.upload_tree(meta, geom, sim.tree.min_lvl, sim.tree.max_lvl, levels)
    for iv in range(N_VAR_CELL):
        r.set_cc(iv, src.cc(iv))
    for d in range(2):
        for f in range(N_VAR_FACE):
            r.set_fc(d, f, src.fc(d, f))
    if mixed:
        r.set_precision(True, schedule)
    return r
