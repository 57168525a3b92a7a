"""Helpers shared by the parity tests: mirror an oracle run onto the device
and compare states. The oracle is the checker here, never the product."""
from __future__ import annotations

import numpy as np

import a5ref
from a5_streamer_b200 import device as dv

N_CC, N_FC = 9, 2


def side_mask(meta: np.ndarray, nc: int) -> np.ndarray:
    """Per-id slot mask of interior + side-ghost cells (corners excluded),
    for each box's own (n_cell+2)^2 layout."""
    S = (nc + 2) ** 2
    mask = np.zeros((meta.shape[0], S), dtype=bool)
    for id_ in range(1, meta.shape[0]):
        if not meta[id_, 0]:
            continue
        n = meta[id_, 14]
        g = n + 2
        m = np.ones((g, g), dtype=bool)
        m[0, 0] = m[0, g - 1] = m[g - 1, 0] = m[g - 1, g - 1] = False
        mask[id_, :g * g] = m.reshape(-1)
    return mask


def interior_mask(meta: np.ndarray, nc: int) -> np.ndarray:
    S = (nc + 2) ** 2
    mask = np.zeros((meta.shape[0], S), dtype=bool)
    for id_ in range(1, meta.shape[0]):
        if not meta[id_, 0]:
            continue
        n = meta[id_, 14]
        g = n + 2
        m = np.zeros((g, g), dtype=bool)
        m[1:n + 1, 1:n + 1] = True
        mask[id_, :g * g] = m.reshape(-1)
    return mask


def face_mask(meta: np.ndarray, nc: int) -> np.ndarray:
    S = (nc + 1) * nc
    mask = np.zeros((meta.shape[0], S), dtype=bool)
    for id_ in range(1, meta.shape[0]):
        if meta[id_, 0]:
            n = meta[id_, 14]
            mask[id_, :(n + 1) * n] = True
    return mask


def device_from_oracle(sim: a5ref.Sim, cfg, run: dv.DeviceRun | None = None) -> dv.DeviceRun:
    """Create (or refresh) a device run holding the oracle's tree, table and data."""
    if run is None:
        run = dv.DeviceRun(cfg)
        rc, xmin, inv = sim.table()
        run.set_table(rc, xmin, inv)
    run.upload_tree(sim.meta(), sim.geom(), sim.min_lvl, sim.max_lvl, sim.levels())
    for iv in range(N_CC):
        run.set_cc(iv, sim.cc(iv))
    for d in range(2):
        for f in range(N_FC):
            run.set_fc(d, f, sim.fc(d, f))
    return run


def compare(sim: a5ref.Sim, run: dv.DeviceRun, cc_vars=range(N_CC), fc_vars=((0, 0), (0, 1), (1, 0), (1, 1)),
            rtol: float = 0.0, mask_kind: str = "side", where: str = ""):
    """Assert device == oracle on the given variables. rtol = 0: bit-exact."""
    meta = sim.meta()
    nc = sim.nc
    mask = side_mask(meta, nc) if mask_kind == "side" else interior_mask(meta, nc)
    fmask = face_mask(meta, nc)
    imask = interior_mask(meta, nc)
    for iv in cc_vars:
        a, b = sim.cc(iv), run.cc(iv)
        # rhs ghost cells are never read by any operator and are not maintained
        m = imask if iv == 6 else mask
        _check(a[m], b[m], rtol, f"{where} cc var {iv}")
    for d, f in fc_vars:
        a, b = sim.fc(d, f), run.fc(d, f)
        _check(a[fmask], b[fmask], rtol, f"{where} face dim {d} var {f}")


def _check(a, b, rtol, what):
    if rtol == 0.0:
        bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
        if bad.any():
            k = np.flatnonzero(bad)
            raise AssertionError(f"{what}: {bad.sum()} of {a.size} values differ; first at {k[:5]}: "
                                 f"oracle {a[k[:5]]} device {b[k[:5]]}")
    else:
        scale = np.maximum(np.abs(a), np.abs(b))
        err = np.abs(a - b)
        bad = err > rtol * np.maximum(scale, 1e-300)
        if bad.any():
            k = np.flatnonzero(bad)
            raise AssertionError(f"{what}: {bad.sum()} of {a.size} values beyond rtol {rtol}; "
                                 f"max rel {np.max(err[bad] / scale[bad]):.3e}")
