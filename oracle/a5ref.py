"""ctypes wrapper of the CPU oracle (test infrastructure only).

The oracle is a plain C++ restatement of the reference's Fortran algorithm,
built into oracle/liba5ref.so by oracle/Makefile. Only the tests, the smoke
check and the CPU-baseline leg of the benchmark use it, as the checker or as
the timed CPU baseline; the product never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liba5ref.so")

MAX_SEEDS = 8
MAX_TD = 4096
TD_COLUMNS = ("mobility", "diffusion", "alpha", "eta")

# variable indices (src/m_streamer.f90:17-43), 0-based
I_ELEC, I_PION, I_ELEC_OLD, I_PION_OLD, I_PHI, I_FLD, I_RHS, I_PHO, I_EPS = range(9)
F_ELEC, F_FLD = 0, 1


class Params(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int), ("coord", ctypes.c_int), ("box_size", ctypes.c_int),
        ("n_base", ctypes.c_int * 3), ("dr_base", ctypes.c_double),
        ("lvls_max", ctypes.c_int), ("domain_len_z", ctypes.c_double),
        ("applied_fld", ctypes.c_double), ("epsilon_diel", ctypes.c_double),
        ("bg_dens", ctypes.c_double), ("n_seeds", ctypes.c_int),
        ("seed_r0", (ctypes.c_double * 3) * MAX_SEEDS),
        ("seed_r1", (ctypes.c_double * 3) * MAX_SEEDS),
        ("seed_dens", ctypes.c_double * MAX_SEEDS),
        ("seed_width", ctypes.c_double * MAX_SEEDS),
        ("seed_falloff", ctypes.c_int * MAX_SEEDS),
        ("dt_max", ctypes.c_double), ("num_steps_amr", ctypes.c_int),
        ("use_drt", ctypes.c_int), ("n_cycle_base", ctypes.c_int),
        ("ref_init_time", ctypes.c_double), ("crv_refine", ctypes.c_double),
        ("lkptbl_size", ctypes.c_int), ("lkptbl_max_fld", ctypes.c_double),
        ("td_n", ctypes.c_int * 4),
        ("td_x", (ctypes.c_double * MAX_TD) * 4),
        ("td_y", (ctypes.c_double * MAX_TD) * 4),
        ("n_threads", ctypes.c_int),
        ("photoi_enabled", ctypes.c_int), ("photoi_num_photons", ctypes.c_int),
        ("photoi_team", ctypes.c_int), ("photoi_tbl_kind", ctypes.c_int),
        ("photoi_coeff", ctypes.c_double), ("photoi_p_O2", ctypes.c_double),
        ("photoi_len_lo", ctypes.c_double), ("photoi_len_hi", ctypes.c_double),
        ("photoi_max_dist", ctypes.c_double), ("photoi_fac_dx", ctypes.c_double),
        ("rng_seed", ctypes.c_int * 4),
        ("uniform_lvl", ctypes.c_int),
    ]


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("a5ref.cpp", "a5ref3.inc", "a5ref.h")]
    if (force or not os.path.exists(LIB_PATH)
            or any(os.path.getmtime(LIB_PATH) < os.path.getmtime(f) for f in srcs)):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        P, D, I, V = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, None
        pd, pi = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        sig = {
            "a5ref_create": (P, [ctypes.POINTER(Params)]), "a5ref_destroy": (V, [P]),
            "a5ref_init": (I, [P]), "a5ref_set_init_cond": (V, [P]),
            "a5ref_get_max_dt": (D, [P]), "a5ref_dt_reductions": (V, [P, pd]),
            "a5ref_step": (V, [P, D]), "a5ref_advance": (D, [P, I]),
            "a5ref_run": (I, [P, D, I]), "a5ref_time": (D, [P]), "a5ref_set_time": (V, [P, D]),
            "a5ref_op_copy_cc": (V, [P, I, I]), "a5ref_op_fluxes_koren": (V, [P, D]),
            "a5ref_op_consistent_fluxes": (V, [P]), "a5ref_op_update_solution": (V, [P, D]),
            "a5ref_op_restrict_tree": (V, [P, I]), "a5ref_op_gc_tree": (V, [P, I, I]),
            "a5ref_op_average_dens": (V, [P]), "a5ref_op_compute_fld": (V, [P, I]),
            "a5ref_op_set_rhs": (V, [P]), "a5ref_op_fmg": (V, [P, I, I]),
            "a5ref_op_fld_from_pot": (V, [P]), "a5ref_op_ref_flags": (V, [P, pi]),
            "a5ref_op_vcycle": (V, [P, I, I]),
            "a5ref_tree_max_cc": (D, [P, I]), "a5ref_tree_min_cc": (D, [P, I]),
            "a5ref_tree_sum_cc": (D, [P, I, I]),
            "a5ref_photons_created": (ctypes.c_longlong, [P]),
            "a5ref_set_level_set": (V, [P, pd, pd]),
            "a5ref_streamer_properties": (V, [P, pd]),
            "a5ref_cc_axis": (I, [P, pd, I]),
            "a5ref_vtk_arrays": (I, [P, I, pi, I, pi, pd, pi, pi, pi, pd]),
            "a5ref_op_regrid": (I, [P, pi, pi]),
            "a5ref_max_id": (I, [P]), "a5ref_max_lvl": (I, [P]), "a5ref_min_lvl": (I, [P]),
            "a5ref_n_leaf_cells": (I, [P]), "a5ref_n_cells_all": (I, [P]),
            "a5ref_export_meta": (V, [P, pi]), "a5ref_export_geom": (V, [P, pd]),
            "a5ref_export_levels": (I, [P, pi, pi, I]),
            "a5ref_export_cc": (V, [P, I, pd]), "a5ref_import_cc": (V, [P, I, pd]),
            "a5ref_export_fc": (V, [P, I, I, pd]), "a5ref_import_fc": (V, [P, I, I, pd]),
            "a5ref_import_tree": (I, [P, I, I, I, pi, pd, I, pi, pi]),
            "a5ref_export_table": (V, [P, pd, pd, pd, pi]),
            "a5ref_applied_voltage": (D, [P]),
            "a5ref_kat_mg2_2d": (I, [I, pd, pd, pi]), "a5ref_kat_mg_cyl": (I, [I, pd, pd, pi]),
            "a5ref_kat_mg_cyl_diel": (I, [I, pd, pd, pi]),
            "a5ref_kat_mg3_2d": (I, [I, pd, pd, pi]),
            "a5ref_kat_mgb_2d": (I, [I, I, pd, pd]),
            "a5ref_kat_lookup": (D, [I, I, D, I]), "a5ref_koren_mlim": (D, [D, D]),
            "a5ref_op_photoionization": (V, [P, D, I]),
            "a5ref_rng_get": (V, [P, pi]), "a5ref_rng_set": (V, [P, pi]),
            "a5ref_photon_table": (I, [P, pd, I, pd, pi]),
            "a5ref_kat_photon_table": (I, [I, D, D, D, D, pd, pd]),
            "a5ref_kat_photon_dist": (D, [D, D, I, I]),
            "a5ref_kat_rng": (V, [pi, I, pi]),
            "a5ref_kat_drift_diff": (I, [I, D, I, pd]),
            # differentiation check (a5ref_tl.inc)
            "a5ref_program": (D, [P, I, pd, D, D]),
            "a5ref_tl_program": (D, [P, I, pd, D, D, I, pd, pd, pd]),
            "a5ref_head_profile": (I, [P, D, pd]),
            "a5ref_set_table_rows": (V, [P, pd]), "a5ref_set_applied_fld": (V, [P, D]),
            # the 3D octree form (uniform octrees)
            "a5ref3_create": (P, [ctypes.POINTER(Params)]), "a5ref3_destroy": (V, [P]),
            "a5ref3_init": (I, [P]), "a5ref3_set_init_cond": (V, [P]),
            "a5ref3_dt_reductions": (V, [P, pd]), "a5ref3_get_max_dt": (D, [P]),
            "a5ref3_step": (V, [P, D]), "a5ref3_advance": (D, [P]),
            "a5ref3_time": (D, [P]), "a5ref3_set_time": (V, [P, D]),
            "a5ref3_op_copy_cc": (V, [P, I, I]), "a5ref3_op_fluxes_koren": (V, [P, D]),
            "a5ref3_op_update_solution": (V, [P, D]), "a5ref3_op_restrict_tree": (V, [P, I]),
            "a5ref3_op_gc_tree": (V, [P, I]), "a5ref3_op_average_dens": (V, [P]),
            "a5ref3_op_set_rhs": (V, [P]), "a5ref3_op_compute_fld": (V, [P, I]),
            "a5ref3_op_fmg": (V, [P, I, I]), "a5ref3_op_vcycle": (V, [P, I, I]),
            "a5ref3_op_fld_from_pot": (V, [P]),
            "a5ref3_tree_max_cc": (D, [P, I]), "a5ref3_tree_min_cc": (D, [P, I]),
            "a5ref3_applied_voltage": (D, [P]),
            "a5ref3_max_id": (I, [P]), "a5ref3_max_lvl": (I, [P]), "a5ref3_min_lvl": (I, [P]),
            "a5ref3_n_leaf_cells": (ctypes.c_longlong, [P]),
            "a5ref3_export_meta": (V, [P, pi]), "a5ref3_export_geom": (V, [P, pd]),
            "a5ref3_export_levels": (I, [P, pi, pi, I]),
            "a5ref3_export_cc": (V, [P, I, pd]), "a5ref3_import_cc": (V, [P, I, pd]),
            "a5ref3_export_fc": (V, [P, I, I, pd]), "a5ref3_import_fc": (V, [P, I, I, pd]),
            "a5ref3_export_table": (V, [P, pd, pd, pd, pi]),
            "a5ref3_kat_mg": (I, [I, I, pd, pd]),
            "a5ref3_kat_drift_diff": (I, [I, D, pd]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def make_params(cfg, n_threads: int = 0) -> Params:
    """Fill the oracle's parameter block from a StreamerConfig-like object."""
    p = Params()
    p.dim = cfg.dim
    p.coord = 1 if cfg.coord == "cyl" else 0
    p.box_size = cfg.box_size
    for d in range(cfg.dim):
        p.n_base[d] = cfg.n_base[d]
    p.dr_base = cfg.dr_base
    p.lvls_max = cfg.lvls_max
    p.domain_len_z = cfg.domain_len_z
    p.applied_fld = cfg.applied_fld
    p.epsilon_diel = cfg.epsilon_diel
    p.bg_dens = cfg.bg_dens
    p.n_seeds = len(cfg.seeds)
    for n, s in enumerate(cfg.seeds):
        for d in range(cfg.dim):
            p.seed_r0[n][d] = s.r0[d]
            p.seed_r1[n][d] = s.r1[d]
        p.seed_dens[n] = s.dens
        p.seed_width[n] = s.width
        p.seed_falloff[n] = s.falloff
    p.dt_max = cfg.dt_max
    p.num_steps_amr = cfg.num_steps_amr
    p.use_drt = 1 if cfg.use_drt else 0
    p.n_cycle_base = cfg.n_cycle_base
    p.ref_init_time = cfg.ref_init_time
    p.crv_refine = cfg.crv_refine
    p.lkptbl_size = cfg.lkptbl_size
    p.lkptbl_max_fld = cfg.lkptbl_max_fld
    for c, name in enumerate(TD_COLUMNS):
        xs, ys = cfg.td[name]
        p.td_n[c] = len(xs)
        for k in range(len(xs)):
            p.td_x[c][k] = xs[k]
            p.td_y[c][k] = ys[k]
    p.n_threads = n_threads
    p.photoi_enabled = 1 if cfg.photoi_enabled else 0
    p.photoi_num_photons = cfg.photoi_num_photons
    p.photoi_team = cfg.photoi_team
    kind, a, b = cfg.photoi_table
    p.photoi_tbl_kind = 0 if kind == "air" else 1
    if kind == "air":
        p.photoi_p_O2 = a
    else:
        p.photoi_len_lo, p.photoi_len_hi = a, b
    p.photoi_coeff = cfg.photoi_coeff
    p.photoi_max_dist = cfg.photoi_max_dist
    p.photoi_fac_dx = cfg.photoi_fac_dx
    for i in range(4):
        p.rng_seed[i] = cfg.rng_seed[i]
    p.uniform_lvl = getattr(cfg, "uniform_lvl", 0)
    return p


class Sim:
    """One oracle simulation (tree + fields)."""

    def __init__(self, cfg, n_threads: int = 0):
        self.cfg = cfg
        self._p = make_params(cfg, n_threads)
        self.h = lib().a5ref_create(ctypes.byref(self._p))
        if not self.h:
            raise ValueError("oracle rejected the parameters")
        self.nc = cfg.box_size

    def close(self):
        if self.h:
            lib().a5ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # driver -----------------------------------------------------------------
    def init(self) -> int:
        return lib().a5ref_init(self.h)

    def set_init_cond(self):
        lib().a5ref_set_init_cond(self.h)

    def get_max_dt(self) -> float:
        return lib().a5ref_get_max_dt(self.h)

    def dt_reductions(self) -> np.ndarray:
        out = np.zeros(3)
        lib().a5ref_dt_reductions(self.h, _dp(out))
        return out

    def step(self, dt: float):
        lib().a5ref_step(self.h, dt)

    def advance(self, regrid: bool = True) -> float:
        return lib().a5ref_advance(self.h, 1 if regrid else 0)

    def run(self, t_end: float, max_blocks: int = 1 << 30) -> int:
        return lib().a5ref_run(self.h, t_end, max_blocks)

    @property
    def time(self) -> float:
        return lib().a5ref_time(self.h)

    @time.setter
    def time(self, t: float):
        lib().a5ref_set_time(self.h, t)

    # ops ------------------------------------------------------------------------
    def op(self, name: str, *args):
        return getattr(lib(), "a5ref_op_" + name)(self.h, *args)

    def tree_max_cc(self, iv: int) -> float:
        return lib().a5ref_tree_max_cc(self.h, iv)

    def tree_min_cc(self, iv: int) -> float:
        return lib().a5ref_tree_min_cc(self.h, iv)

    def tree_sum_cc(self, iv: int, team: int = 1) -> float:
        return lib().a5ref_tree_sum_cc(self.h, iv, team)

    def set_level_set(self, lsf, bval):
        if lsf is None:
            lib().a5ref_set_level_set(self.h, None, None)
            return
        lsf = np.ascontiguousarray(lsf, dtype=np.float64)
        bval = np.ascontiguousarray(bval, dtype=np.float64)
        lib().a5ref_set_level_set(self.h, _dp(lsf), _dp(bval))

    def photons_created(self) -> int:
        return int(lib().a5ref_photons_created(self.h))

    def streamer_properties(self) -> np.ndarray:
        """get_streamer_properties restated in the oracle (39 values)."""
        out = np.zeros(39)
        lib().a5ref_streamer_properties(self.h, _dp(out))
        return out

    def vtk_arrays(self, ivs, ifs=()):
        """a$D_write_vtk's arrays restated in the oracle: dict of coords
        (n_nodes x 2), connectivity, offsets, types and the values (one row
        per cell variable, then fx and fy means per face variable)."""
        iv = np.ascontiguousarray(ivs, dtype=np.int32)
        fv = np.ascontiguousarray(ifs if len(ifs) else [0], dtype=np.int32)
        n = lib().a5ref_vtk_arrays(self.h, len(ivs), _ip(iv), len(ifs), _ip(fv), None, None, None,
                                   None, None)
        nodes = (n // (self.nc * self.nc)) * (self.nc + 1) ** 2
        coords = np.zeros(2 * nodes)
        con = np.zeros(4 * n, dtype=np.int32)
        off = np.zeros(n, dtype=np.int32)
        ty = np.zeros(n, dtype=np.int32)
        vals = np.zeros((len(ivs) + 2 * len(ifs), n))
        lib().a5ref_vtk_arrays(self.h, len(ivs), _ip(iv), len(ifs), _ip(fv), _dp(coords), _ip(con),
                               _ip(off), _ip(ty), _dp(vals))
        return {"coords": coords.reshape(-1, 2), "connectivity": con, "offsets": off, "types": ty,
                "values": vals}

    def cc_axis(self) -> np.ndarray:
        """get_cc_axis restated in the oracle: rows z, n_e, n_i, axial field,
        axial electron flux."""
        n = lib().a5ref_cc_axis(self.h, None, 0)
        out = np.zeros(5 * max(n, 1))
        lib().a5ref_cc_axis(self.h, _dp(out), n)
        return out[:5 * n].reshape(5, n)

    def ref_flags(self) -> np.ndarray:
        out = np.zeros(self.max_id + 1, dtype=np.int32)
        lib().a5ref_op_ref_flags(self.h, _ip(out))
        return out

    def regrid(self):
        a, r = ctypes.c_int(0), ctypes.c_int(0)
        lib().a5ref_op_regrid(self.h, ctypes.byref(a), ctypes.byref(r))
        return a.value, r.value

    # tree / data export -------------------------------------------------------
    @property
    def max_id(self) -> int:
        return lib().a5ref_max_id(self.h)

    @property
    def max_lvl(self) -> int:
        return lib().a5ref_max_lvl(self.h)

    @property
    def min_lvl(self) -> int:
        return lib().a5ref_min_lvl(self.h)

    def n_leaf_cells(self) -> int:
        return lib().a5ref_n_leaf_cells(self.h)

    def n_cells_all(self) -> int:
        return lib().a5ref_n_cells_all(self.h)

    def meta(self) -> np.ndarray:
        m = np.zeros((self.max_id + 1, 16), dtype=np.int32)
        lib().a5ref_export_meta(self.h, _ip(m))
        return m

    def geom(self) -> np.ndarray:
        g = np.zeros((self.max_id + 1, 4))
        lib().a5ref_export_geom(self.h, _dp(g))
        return g

    def levels(self):
        nlev = self.max_lvl - self.min_lvl + 1
        counts = np.zeros((nlev, 3), dtype=np.int32)
        cap = 3 * (self.max_id + 1)
        ids = np.zeros(cap, dtype=np.int32)
        lib().a5ref_export_levels(self.h, _ip(counts), _ip(ids), cap)
        out, k = {}, 0
        for li in range(nlev):
            lvl = self.min_lvl + li
            n_ids, n_lv, n_pa = counts[li]
            a = ids[k:k + n_ids].copy(); k += n_ids
            b = ids[k:k + n_lv].copy(); k += n_lv
            c = ids[k:k + n_pa].copy(); k += n_pa
            out[lvl] = (a, b, c)
        return out

    def cc(self, iv: int) -> np.ndarray:
        S = (self.nc + 2) ** 2
        out = np.zeros((self.max_id + 1, S))
        lib().a5ref_export_cc(self.h, iv, _dp(out))
        return out

    def set_cc(self, iv: int, data: np.ndarray):
        data = np.ascontiguousarray(data, dtype=np.float64)
        lib().a5ref_import_cc(self.h, iv, _dp(data))

    def fc(self, dimf: int, f: int) -> np.ndarray:
        S = (self.nc + 1) * self.nc
        out = np.zeros((self.max_id + 1, S))
        lib().a5ref_export_fc(self.h, dimf, f, _dp(out))
        return out

    def set_fc(self, dimf: int, f: int, data: np.ndarray):
        data = np.ascontiguousarray(data, dtype=np.float64)
        lib().a5ref_import_fc(self.h, dimf, f, _dp(data))

    def table(self):
        n = ctypes.c_int(0)
        xm, inv = ctypes.c_double(0), ctypes.c_double(0)
        lib().a5ref_export_table(self.h, None, ctypes.byref(xm), ctypes.byref(inv), ctypes.byref(n))
        rc = np.zeros(n.value * 4)
        lib().a5ref_export_table(self.h, _dp(rc), None, None, None)
        return rc.reshape(4, n.value).T.copy(), xm.value, inv.value

    @property
    def applied_voltage(self) -> float:
        return lib().a5ref_applied_voltage(self.h)

    def photoionization(self, dt: float | None):
        lib().a5ref_op_photoionization(self.h, 0.0 if dt is None else dt, 0 if dt is None else 1)

    # differentiation check (a5ref_tl.inc) ---------------------------------------
    def program(self, dts, x0: float, T: float) -> float:
        """J of the fixed-mesh program: initial conditions, first field solve,
        len(dts) steps, head height at the line x = x0 with softmax temperature T."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        return lib().a5ref_program(self.h, len(d), _dp(d), x0, T)

    def tl_program(self, dts, x0: float, T: float, dtbl, dV):
        """(J, dJ): tangent-linear run along the directions dtbl[k] (derivative
        of the table rows, n_rows x 4) and dV[k] (of the applied voltage)."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        dtbl = np.asarray(dtbl, dtype=np.float64)
        n_dir = dtbl.shape[0]
        dt_cm = np.ascontiguousarray(np.transpose(dtbl, (0, 2, 1)))  # column-major rows
        dv = np.ascontiguousarray(dV, dtype=np.float64)
        dJ = np.zeros(n_dir)
        J = lib().a5ref_tl_program(self.h, len(d), _dp(d), x0, T, n_dir, _dp(dt_cm), _dp(dv),
                                   _dp(dJ))
        return J, dJ

    def head_profile(self, x0: float) -> np.ndarray:
        n = lib().a5ref_head_profile(self.h, x0, None)
        out = np.zeros((max(n, 1), 3))
        lib().a5ref_head_profile(self.h, x0, _dp(out))
        return out[:n]

    def set_table_rows(self, rows: np.ndarray):
        """rows: n_rows x 4 (mobility, diffusion, alpha, eta)."""
        rc = np.ascontiguousarray(np.asarray(rows, dtype=np.float64).T)
        lib().a5ref_set_table_rows(self.h, _dp(rc))

    def set_applied_fld(self, fld: float):
        lib().a5ref_set_applied_fld(self.h, fld)

    def rng_state(self) -> np.ndarray:
        st = np.zeros(4, dtype=np.int32)
        lib().a5ref_rng_get(self.h, _ip(st))
        return st

    def set_rng_state(self, st) -> None:
        st = np.ascontiguousarray(st, dtype=np.int32)
        lib().a5ref_rng_set(self.h, _ip(st))

    # run checkpoints in the product's layout (a5s_checkpoint_save) -------
    _CK_MAGIC, _CK_VERSION = 0x4B433541, 1

    def checkpoint(self) -> bytes:
        """This run's state in the layout of a5s_checkpoint_save (native
        little-endian, fingerprint 0); the level lists above max_lvl, which no
        operation reads before rebuilding them, are written empty."""
        import struct
        nc, M = self.nc, self.max_id + 1
        n_lists = self.cfg.lvls_max + 2 - self.min_lvl
        photoi = 1 if self.cfg.photoi_enabled else 0
        rng = self.rng_state() if photoi else np.zeros(4, dtype=np.int32)
        out = [struct.pack("<IIQ", self._CK_MAGIC, self._CK_VERSION, 0),
               struct.pack("<10i", nc, 1 if self.cfg.coord == "cyl" else 0, self.cfg.lvls_max,
                           self.min_lvl, self.max_lvl, self.max_id, n_lists, (nc + 2) ** 2,
                           (nc + 1) * nc, photoi),
               struct.pack("<d", self.time), rng.astype("<i4").tobytes()]
        meta, geom = self.meta(), self.geom()
        rec = np.zeros(M, dtype=[("i", "<i4", 14), ("d", "<f8", 3)])
        rec["i"][:, 0:4] = meta[:, 0:4]
        rec["i"][:, 4] = meta[:, 5]
        rec["i"][:, 5] = meta[:, 14]
        rec["i"][:, 6:14] = meta[:, 6:14]
        rec["d"][:, 0] = geom[:, 3]
        rec["d"][:, 1:3] = geom[:, 0:2]
        out.append(rec.tobytes())
        levels = self.levels()
        for k in range(n_lists):
            a, b, c = levels.get(self.min_lvl + k, ([], [], []))
            out.append(struct.pack("<3i", len(a), len(b), len(c)))
            out.append(np.concatenate([np.asarray(x, dtype="<i4") for x in (a, b, c)]).tobytes())
        for iv in range(9):
            out.append(self.cc(iv).astype("<f8").tobytes())
        for d in range(2):
            for f in range(2):
                out.append(self.fc(d, f).astype("<f8").tobytes())
        return b"".join(out)

    def load_checkpoint(self, buf: bytes) -> None:
        """Resume from a checkpoint in the layout of a5s_checkpoint_save, for
        instance one the device path wrote (the fingerprint is not checked)."""
        import struct
        magic, version, _ = struct.unpack_from("<IIQ", buf, 0)
        if (magic, version) != (self._CK_MAGIC, self._CK_VERSION):
            raise ValueError("not a checkpoint of this layout")
        nc, _coord, _lm, min_lvl, max_lvl, max_id, n_lists, cslot, fslot, photoi = \
            struct.unpack_from("<10i", buf, 16)
        if nc != self.nc or cslot != (nc + 2) ** 2 or fslot != (nc + 1) * nc:
            raise ValueError("checkpoint of another box size")
        (t,) = struct.unpack_from("<d", buf, 56)
        rng = np.frombuffer(buf, dtype="<i4", count=4, offset=64)
        off = 80
        M = max_id + 1
        rec = np.frombuffer(buf, dtype=[("i", "<i4", 14), ("d", "<f8", 3)], count=M, offset=off)
        off += rec.itemsize * M
        counts, ids = [], []
        for _ in range(n_lists):
            a, b, c = struct.unpack_from("<3i", buf, off)
            off += 12
            counts += [a, b, c]
            ids.append(np.frombuffer(buf, dtype="<i4", count=a + b + c, offset=off))
            off += 4 * (a + b + c)
        ri = np.ascontiguousarray(rec["i"], dtype=np.int32)
        rd = np.ascontiguousarray(rec["d"], dtype=np.float64)
        cnt = np.asarray(counts, dtype=np.int32)
        idv = np.ascontiguousarray(np.concatenate(ids + [np.zeros(1, dtype="<i4")]), dtype=np.int32)
        if lib().a5ref_import_tree(self.h, max_id, min_lvl, max_lvl, _ip(ri), _dp(rd), n_lists,
                                   _ip(cnt), _ip(idv)) != 0:
            raise ValueError("checkpoint tree does not fit this run")
        for iv in range(9):
            x = np.frombuffer(buf, dtype="<f8", count=M * cslot, offset=off)
            off += 8 * M * cslot
            self.set_cc(iv, x.reshape(M, cslot))
        for d in range(2):
            for f in range(2):
                x = np.frombuffer(buf, dtype="<f8", count=M * fslot, offset=off)
                off += 8 * M * fslot
                self.set_fc(d, f, x.reshape(M, fslot))
        if off != len(buf):
            raise ValueError("checkpoint length does not match its header")
        self.time = t
        if photoi:
            self.set_rng_state(rng)

    def photon_table(self):
        """(distances at the table's cumulative fractions, frac_in_tbl, absorption level)"""
        frac, lvl = ctypes.c_double(0), ctypes.c_int(0)
        n = lib().a5ref_photon_table(self.h, None, 0, ctypes.byref(frac), ctypes.byref(lvl))
        d = np.zeros(max(n, 1))
        lib().a5ref_photon_table(self.h, _dp(d), n, None, None)
        return d[:n], frac.value, lvl.value


def kat_mg(cyl: bool, n_fmg: int):
    res, err = np.zeros(n_fmg), np.zeros(n_fmg)
    ml = ctypes.c_int(0)
    fn = lib().a5ref_kat_mg_cyl if cyl else lib().a5ref_kat_mg2_2d
    cells = fn(n_fmg, _dp(res), _dp(err), ctypes.byref(ml))
    return res, err, ml.value, cells


def kat_mg_diel(n_fmg: int):
    """The dielectric multigrid case (test_mg_cyl_diel.f90): per FMG cycle max
    |residual| and max |error|, the finest level and the number of boxes the
    multigrid treats as dielectric."""
    res, err = np.zeros(n_fmg), np.zeros(n_fmg)
    ml = ctypes.c_int(0)
    n_diel = lib().a5ref_kat_mg_cyl_diel(n_fmg, _dp(res), _dp(err), ctypes.byref(ml))
    return res, err, ml.value, n_diel


def kat_mg3_2d(n_fmg: int):
    """The layered dielectric case (test_mg3_2d.f90): per FMG cycle max
    |residual| and max |error| against the piecewise-linear solution, the
    finest level and the number of leaf boxes."""
    res, err = np.zeros(n_fmg), np.zeros(n_fmg)
    ml = ctypes.c_int(0)
    n = lib().a5ref_kat_mg3_2d(n_fmg, _dp(res), _dp(err), ctypes.byref(ml))
    return res, err, ml.value, n


def kat_mgb_2d(shape: str, n_fmg: int):
    """The level-set boundary case (test_mgb_2d.f90; 'ellipse' or 'plane'):
    per FMG cycle max |residual| and max |error| (plane), and the number of
    boxes tagged for the level-set operators."""
    res, err = np.zeros(n_fmg), np.zeros(n_fmg)
    n = lib().a5ref_kat_mgb_2d(0 if shape == "ellipse" else 1, n_fmg, _dp(res), _dp(err))
    return res, err, n


def kat_lookup(n_rows: int, n_pairs: int = 100000, x_max: float = 10.0,
               n_samples: int = 10000) -> float:
    return lib().a5ref_kat_lookup(n_rows, n_pairs, x_max, n_samples)


def koren_mlim(a: float, b: float) -> float:
    return lib().a5ref_koren_mlim(a, b)


def kat_photon_table(kind: str, a: float, b: float, max_dist: float):
    d = np.zeros(500)
    frac = ctypes.c_double(0)
    n = lib().a5ref_kat_photon_table(0 if kind == "air" else 1, a if kind == "air" else 0.0,
                                     a if kind != "air" else 0.0, b if kind != "air" else 0.0,
                                     max_dist, _dp(d), ctypes.byref(frac))
    if n < 0:
        raise ValueError("photon table integration failed")
    return d[:n], frac.value


def kat_photon_dist(p_O2: float, max_dist: float, n_photons: int, n_team: int) -> float:
    return lib().a5ref_kat_photon_dist(p_O2, max_dist, n_photons, n_team)


def kat_rng(state4, n: int) -> np.ndarray:
    st = np.ascontiguousarray(state4, dtype=np.int32)
    out = np.zeros(n, dtype=np.int32)
    lib().a5ref_kat_rng(_ip(st), n, _ip(out))
    return out


def kat_drift_diff(uniform_lvl: int = 0, end_time: float = 5.0, regrid: bool = True) -> dict:
    """The drift-diffusion example (afivo/examples/transport/
    test_drift_diff_2d.f90) on the oracle's transport machinery: errors
    against the exact advected solution and the conserved sum of phi."""
    out = np.zeros(8)
    rc = lib().a5ref_kat_drift_diff(uniform_lvl, end_time, 1 if regrid else 0, _dp(out))
    if rc != 0:
        raise RuntimeError("drift-diffusion case touched a physical boundary")
    keys = ("max_err", "mean_err", "sum0", "sum_end", "steps", "max_lvl", "leaf_cells", "time")
    return dict(zip(keys, out.tolist()))


class Sim3:
    """One oracle simulation of the 3D octree form (a uniformly refined
    octree; src/streamer_3d.f90 with afivo's m_a3_* routines)."""

    def __init__(self, cfg, n_threads: int = 0):
        self.cfg = cfg
        self._p = make_params(cfg, n_threads)
        self.h = lib().a5ref3_create(ctypes.byref(self._p))
        if not self.h:
            raise ValueError("oracle rejected the 3D parameters")
        self.nc = cfg.box_size

    def close(self):
        if self.h:
            lib().a5ref3_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self) -> int:
        it = lib().a5ref3_init(self.h)
        if it < 0:
            raise RuntimeError("3D oracle: tree construction failed")
        return it

    def set_init_cond(self):
        lib().a5ref3_set_init_cond(self.h)

    def get_max_dt(self) -> float:
        return lib().a5ref3_get_max_dt(self.h)

    def dt_reductions(self) -> np.ndarray:
        out = np.zeros(3)
        lib().a5ref3_dt_reductions(self.h, _dp(out))
        return out

    def step(self, dt: float):
        lib().a5ref3_step(self.h, dt)

    def advance(self) -> float:
        return lib().a5ref3_advance(self.h)

    @property
    def time(self) -> float:
        return lib().a5ref3_time(self.h)

    @time.setter
    def time(self, t: float):
        lib().a5ref3_set_time(self.h, t)

    def op(self, name: str, *args):
        return getattr(lib(), "a5ref3_op_" + name)(self.h, *args)

    def tree_max_cc(self, iv: int) -> float:
        return lib().a5ref3_tree_max_cc(self.h, iv)

    def tree_min_cc(self, iv: int) -> float:
        return lib().a5ref3_tree_min_cc(self.h, iv)

    @property
    def max_id(self) -> int:
        return lib().a5ref3_max_id(self.h)

    @property
    def max_lvl(self) -> int:
        return lib().a5ref3_max_lvl(self.h)

    @property
    def min_lvl(self) -> int:
        return lib().a5ref3_min_lvl(self.h)

    def n_leaf_cells(self) -> int:
        return lib().a5ref3_n_leaf_cells(self.h)

    def meta(self) -> np.ndarray:
        m = np.zeros((self.max_id + 1, 24), dtype=np.int32)
        lib().a5ref3_export_meta(self.h, _ip(m))
        return m

    def geom(self) -> np.ndarray:
        g = np.zeros((self.max_id + 1, 4))
        lib().a5ref3_export_geom(self.h, _dp(g))
        return g

    def levels(self):
        nlev = self.max_lvl - self.min_lvl + 1
        counts = np.zeros((nlev, 3), dtype=np.int32)
        cap = 3 * (self.max_id + 1)
        ids = np.zeros(cap, dtype=np.int32)
        lib().a5ref3_export_levels(self.h, _ip(counts), _ip(ids), cap)
        out, k = {}, 0
        for li in range(nlev):
            n_ids, n_lv, n_pa = counts[li]
            a = ids[k:k + n_ids].copy(); k += n_ids
            b = ids[k:k + n_lv].copy(); k += n_lv
            c = ids[k:k + n_pa].copy(); k += n_pa
            out[self.min_lvl + li] = (a, b, c)
        return out

    def cc(self, iv: int) -> np.ndarray:
        out = np.zeros((self.max_id + 1, (self.nc + 2) ** 3))
        lib().a5ref3_export_cc(self.h, iv, _dp(out))
        return out

    def set_cc(self, iv: int, data: np.ndarray):
        data = np.ascontiguousarray(data, dtype=np.float64)
        lib().a5ref3_import_cc(self.h, iv, _dp(data))

    def fc(self, dimf: int, f: int) -> np.ndarray:
        out = np.zeros((self.max_id + 1, (self.nc + 1) * self.nc * self.nc))
        lib().a5ref3_export_fc(self.h, dimf, f, _dp(out))
        return out

    def set_fc(self, dimf: int, f: int, data: np.ndarray):
        data = np.ascontiguousarray(data, dtype=np.float64)
        lib().a5ref3_import_fc(self.h, dimf, f, _dp(data))

    def table(self):
        n_rows = ctypes.c_int()
        x_min, inv_dx = ctypes.c_double(), ctypes.c_double()
        lib().a5ref3_export_table(self.h, None, ctypes.byref(x_min), ctypes.byref(inv_dx),
                                  ctypes.byref(n_rows))
        rc = np.zeros(n_rows.value * 4)
        lib().a5ref3_export_table(self.h, _dp(rc), None, None, None)
        return rc, x_min.value, inv_dx.value, n_rows.value

    @property
    def applied_voltage(self) -> float:
        return lib().a5ref3_applied_voltage(self.h)


def kat_mg3(level: int, n_fmg: int):
    """test_mg2_3d on a uniform octree: max |residual| and max |error| after
    each FMG cycle."""
    res, err = np.zeros(n_fmg), np.zeros(n_fmg)
    lvl = lib().a5ref3_kat_mg(level, n_fmg, _dp(res), _dp(err))
    if lvl < 0:
        raise RuntimeError("3D multigrid case failed")
    return res, err


def kat_drift_diff3(level: int, end_time: float = 1.0) -> dict:
    """test_drift_diff_3d on a uniform octree: errors against the exact
    advected solution and the conserved sum of phi."""
    out = np.zeros(8)
    rc = lib().a5ref3_kat_drift_diff(level, end_time, _dp(out))
    if rc != 0:
        raise RuntimeError("3D drift-diffusion case failed")
    keys = ("max_err", "mean_err", "sum0", "sum_end", "steps", "max_lvl", "leaf_cells", "time")
    return dict(zip(keys, out.tolist()))
