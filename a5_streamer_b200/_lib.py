"""ctypes binding of the C ABI declared in include/a5g.h.

The library is loaded from the package directory; if it is missing the import
raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liba5g.so")

A5G_OK, A5G_EINVAL, A5G_ENOMEM, A5G_ECUDA, A5G_TIMEOUT, A5G_ENONFINITE, A5G_ESTATE = range(7)
STATUS_NAMES = {0: "A5G_OK", 1: "A5G_EINVAL", 2: "A5G_ENOMEM", 3: "A5G_ECUDA",
                4: "A5G_TIMEOUT", 5: "A5G_ENONFINITE", 6: "A5G_ESTATE"}


class A5GError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [
        ("box_size", ctypes.c_int), ("coord", ctypes.c_int), ("lvls_max", ctypes.c_int),
        ("dr_base", ctypes.c_double), ("domain_len_z", ctypes.c_double),
        ("applied_fld", ctypes.c_double), ("epsilon_diel", ctypes.c_double),
        ("dt_max", ctypes.c_double), ("use_drt", ctypes.c_int), ("n_cycle_base", ctypes.c_int),
        ("ref_init_time", ctypes.c_double), ("crv_refine", ctypes.c_double),
        ("n_seeds", ctypes.c_int),
        ("seed_r0", (ctypes.c_double * 2) * 8), ("seed_r1", (ctypes.c_double * 2) * 8),
        ("seed_width", ctypes.c_double * 8),
        ("photoi_enabled", ctypes.c_int), ("photoi_num_photons", ctypes.c_int),
        ("photoi_team", ctypes.c_int), ("photoi_pad", ctypes.c_int),
        ("photoi_coeff", ctypes.c_double), ("photoi_fac_dx", ctypes.c_double),
        ("rng_seed", ctypes.c_int * 4),
        ("uniform_lvl", ctypes.c_int), ("uniform_pad", ctypes.c_int),
    ]


A5G_FP64, A5G_MIXED = 0, 1


class MGSchedule(ctypes.Structure):
    """a5g_mg_schedule: multigrid schedule of the FP32 correction solve."""
    _fields_ = [("fmg", ctypes.c_int), ("n_cycle_down", ctypes.c_int),
                ("n_cycle_up", ctypes.c_int), ("n_cycle_base", ctypes.c_int),
                ("n_corr", ctypes.c_int)]


# name -> (restype, argtypes); every function returns an a5g_status int
_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_PD = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)
SIGNATURES = {
    "a5g_last_error": (ctypes.c_char_p, []),
    "a5g_version": (_I, []),
    "a5g_create": (_I, [ctypes.POINTER(Params), ctypes.POINTER(_P)]),
    "a5g_destroy": (_I, [_P]),
    "a5g_set_table": (_I, [_P, _I, _I, _D, _D, _PD]),
    "a5g_upload_tree": (_I, [_P, _I, _I, _I, _PI, _PD, _PI, _PI]),
    "a5g_upload_cc": (_I, [_P, _I, _PD]),
    "a5g_download_cc": (_I, [_P, _I, _PD]),
    "a5g_upload_fc": (_I, [_P, _I, _I, _PD]),
    "a5g_download_fc": (_I, [_P, _I, _I, _PD]),
    "a5g_tree_copy_cc": (_I, [_P, _I, _I]),
    "a5g_fluxes_koren": (_I, [_P, _D]),
    "a5g_consistent_fluxes": (_I, [_P]),
    "a5g_update_solution": (_I, [_P, _D]),
    "a5g_restrict_tree": (_I, [_P, _I]),
    "a5g_gc_tree": (_I, [_P, _I, _I]),
    "a5g_average_dens": (_I, [_P]),
    "a5g_compute_fld": (_I, [_P, _I]),
    "a5g_compute_fld_fp64": (_I, [_P, _I]),
    "a5g_fas_fmg": (_I, [_P, _I, _I]),
    "a5g_fld_from_pot": (_I, [_P]),
    "a5g_mg_fas_vcycle": (_I, [_P, _I, _I]),
    "a5g_tree_max_cc": (_I, [_P, _I, _PD]),
    "a5g_tree_min_cc": (_I, [_P, _I, _PD]),
    "a5g_tree_sum_cc": (_I, [_P, _I, _I, _PD]),
    "a5g_dt_reductions": (_I, [_P, _PD]),
    "a5g_get_max_dt": (_I, [_P, _PD]),
    "a5g_ref_flags": (_I, [_P, _D, _PI]),
    "a5g_prolong_new": (_I, [_P, _PI, _PI]),
    "a5g_step": (_I, [_P, _D]),
    "a5g_set_precision": (_I, [_P, _I, ctypes.POINTER(MGSchedule)]),
    "a5g_get_precision": (_I, [_P, _PI, ctypes.POINTER(MGSchedule)]),
    "a5g_set_photon_table": (_I, [_P, _I, _D, _D, _PD, _D]),
    "a5g_get_rng": (_I, [_P, _PI]),
    "a5g_set_rng": (_I, [_P, _PI]),
    "a5g_photoionization": (_I, [_P, _D, _I]),
    "a5g_photon_stats": (_I, [_P, ctypes.POINTER(ctypes.c_longlong), _PD]),
    "a5g_step_batch": (_I, [ctypes.POINTER(_P), _I, _PD]),
    "a5g_step_batch_static": (_I, [ctypes.POINTER(_P), _I, _PD]),
    "a5g_sync": (_I, [_P]),
    "a5g_set_ctas": (_I, [_P, _I, ctypes.c_longlong]),
    "a5g_get_ctas": (_I, [_P, _PI, _PI]),
    "a5g_set_grid_local": (_I, [_P, _I]),
    "a5g_set_level_set": (_I, [_P, _PD, _PD]),
    "a5g_batch_create": (_I, [ctypes.POINTER(_P), _I, ctypes.POINTER(_P)]),
    "a5g_batch_destroy": (_I, [_P]),
    "a5g_batch_begin": (_I, [_P, _PD, _PD]),
    "a5g_batch_block": (_I, [_P, _I, _I, _PD, _PD, _PI, ctypes.POINTER(ctypes.c_float)]),
    "a5g_n_leaf_cells": (_I, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    "a5g_get_stream": (_I, [_P, ctypes.POINTER(_P)]),
    "a5g_debug_set_staging": (_I, [_P, _I]),
    "a5g_debug_info": (_I, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    "a5g_debug_params_layout": (_I, [_PI, _I]),
    "a5g_debug_plans": (_I, [_I, _I, _I, _PI, _PD, _PI, _PI, _D, _PI, _PI, _P, _PI, _PD, _PI]),
    # host tree (include/a5t.h)
    "a5t_create": (_I, [_I, _I, _D, _PD, _I, ctypes.POINTER(_P)]),
    "a5t_destroy": (_I, [_P]),
    "a5t_set_base": (_I, [_P, _I, _PI, _PI]),
    "a5t_adjust_refinement": (_I, [_P, _PI, _PI, _PI]),
    "a5t_max_id": (_I, [_P]),
    "a5t_min_lvl": (_I, [_P]),
    "a5t_max_lvl": (_I, [_P]),
    "a5t_export": (_I, [_P, _PI, _PD, _PI, _PI]),
    "a5t_n_level_ids": (_I, [_P]),
    "a5t_new_boxes": (_I, [_P, _PI, _PI]),
    "a5t_photon_table": (_I, [_I, _D, _D, _D, _PD, _PD, _PI]),
    # streamer driver
    "a5s_create": (_I, [ctypes.c_void_p, ctypes.POINTER(_P)]),
    "a5s_destroy": (_I, [_P]),
    "a5s_init": (_I, [_P, _PI]),
    "a5s_advance": (_I, [_P, _I, _PD]),
    "a5s_run": (_I, [_P, _D, _I, _PI]),
    "a5s_time": (_I, [_P, _PD]),
    "a5s_batch_run": (_I, [ctypes.POINTER(_P), _I, _PD, _I, _I, _I, _I, _PI, _PD, _PD, _PD]),
    "a5g_batch_launch": (_I, [_P, _I, _I]),
    "a5g_batch_finish": (_I, [_P, _PD, _PD, _PI, ctypes.POINTER(ctypes.c_float)]),
    "a5s_ctx": (_I, [_P, ctypes.POINTER(_P)]),
    "a5s_tree": (_I, [_P, ctypes.POINTER(_P)]),
    "a5s_table": (_I, [_P, _PD, _PD, _PD, _PI]),
}


class Params3(ctypes.Structure):
    """a5g3_params (include/a5g3.h)."""
    _fields_ = [
        ("box_size", ctypes.c_int), ("n_base", ctypes.c_int * 3), ("uniform_lvl", ctypes.c_int),
        ("n_cycle_base", ctypes.c_int), ("use_drt", ctypes.c_int), ("pad", ctypes.c_int),
        ("dr_base", ctypes.c_double), ("domain_len_z", ctypes.c_double),
        ("applied_fld", ctypes.c_double), ("dt_max", ctypes.c_double),
    ]


_PP = ctypes.POINTER(ctypes.c_void_p)
_LL = ctypes.c_longlong
SIGNATURES.update({
    "a5g3_last_error": (ctypes.c_char_p, []),
    "a5g3_create": (_I, [ctypes.POINTER(Params3), _PP]),
    "a5g3_destroy": (_I, [_P]),
    "a5g3_info": (_I, [_P, _PI, _PI, _PI, ctypes.POINTER(_LL)]),
    "a5g3_export_meta": (_I, [_P, _PI]),
    "a5g3_export_levels": (_I, [_P, _PI, _PI, _I, _PI]),
    "a5g3_set_table": (_I, [_P, _I, _I, _D, _D, _PD]),
    "a5g3_set_init_cond": (_I, [_P, _D, _I, _PD, _PD, _PD, _PD, _PI]),
    "a5g3_upload_cc": (_I, [_P, _I, _PD]), "a5g3_download_cc": (_I, [_P, _I, _PD]),
    "a5g3_upload_fc": (_I, [_P, _I, _I, _PD]), "a5g3_download_fc": (_I, [_P, _I, _I, _PD]),
    "a5g3_tree_copy_cc": (_I, [_P, _I, _I]),
    "a5g3_fluxes_koren": (_I, [_P, _D]), "a5g3_update_solution": (_I, [_P, _D]),
    "a5g3_restrict_tree": (_I, [_P, _I]), "a5g3_gc_tree": (_I, [_P, _I]),
    "a5g3_average_dens": (_I, [_P]), "a5g3_compute_fld": (_I, [_P, _I]),
    "a5g3_fmg": (_I, [_P, _I, _I]), "a5g3_vcycle": (_I, [_P, _I, _I]),
    "a5g3_set_rhs": (_I, [_P]), "a5g3_fld_from_pot": (_I, [_P]),
    "a5g3_tree_max_cc": (_I, [_P, _I, _PD]), "a5g3_tree_min_cc": (_I, [_P, _I, _PD]),
    "a5g3_dt_reductions": (_I, [_P, _PD]), "a5g3_get_max_dt": (_I, [_P, _PD]),
    "a5g3_step": (_I, [_P, _D]), "a5g3_sync": (_I, [_P]),
    "a5g3_set_precision": (_I, [_P, _I, ctypes.POINTER(MGSchedule)]),
    "a5g3_get_precision": (_I, [_P, _PI, ctypes.POINTER(MGSchedule)]),
    "a5g3_stream": (_I, [_P, _PP]),
})


class AdjParams(ctypes.Structure):
    """a5a_params (include/a5a.h)."""
    _fields_ = [("n_steps", ctypes.c_int), ("checkpoint_every", ctypes.c_int),
                ("x0", ctypes.c_double), ("temperature", ctypes.c_double)]


_PU = ctypes.POINTER(ctypes.c_uint)
SIGNATURES.update({
    # adjoint (include/a5a.h)
    "a5a_create": (_I, [_P, ctypes.POINTER(AdjParams), _PD, _PP]),
    "a5a_destroy": (_I, [_P]),
    "a5a_forward": (_I, [_P, _PD]),
    "a5a_gradient": (_I, [_P, _PD, _PD, _PD]),
    "a5a_debug_tape": (_I, [_I, _I, _I, _PI, _PD, _PI, _PI, _I, _I, _I,
                            ctypes.POINTER(ctypes.c_longlong), _PI, _PU, _PD, _PI, _PU, _PD]),
    "a5g_set_applied_field": (_I, [_P, _D]),
    "a5s_set_init_cond": (_I, [_P]),
    "a5t_check": (_I, [_P]),
    # checkpoint / resume (include/a5t.h)
    "a5s_checkpoint_size": (_I, [_P, ctypes.POINTER(ctypes.c_size_t)]),
    "a5s_checkpoint_save": (_I, [_P, ctypes.c_void_p, ctypes.c_size_t,
                                 ctypes.POINTER(ctypes.c_size_t)]),
    "a5s_checkpoint_load": (_I, [_P, ctypes.c_void_p, ctypes.c_size_t]),
})


class SimConfig(ctypes.Structure):
    _fields_ = [
        ("dev", Params), ("n_base", ctypes.c_int * 2), ("bg_dens", ctypes.c_double),
        ("n_seeds", ctypes.c_int), ("seed_dens", ctypes.c_double * 8),
        ("seed_falloff", ctypes.c_int * 8), ("num_steps_amr", ctypes.c_int),
        ("lkptbl_size", ctypes.c_int), ("lkptbl_max_fld", ctypes.c_double),
        ("td_n", ctypes.c_int * 4), ("td_x", _PD * 4), ("td_y", _PD * 4),
        ("photoi_tbl_kind", ctypes.c_int), ("photoi_tbl_a", ctypes.c_double),
        ("photoi_tbl_b", ctypes.c_double), ("photoi_max_dist", ctypes.c_double),
    ]

_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              "`python -m a5_streamer_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != A5G_OK:
        msg = lib().a5g_last_error()
        raise A5GError(code, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def check3(code: int) -> None:
    if code != A5G_OK:
        msg = lib().a5g3_last_error()
        raise A5GError(code, msg.decode() if msg else "")


def call3(name: str, *args) -> None:
    check3(getattr(lib(), name)(*args))
