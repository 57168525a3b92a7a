"""Autotuner of the mixed-precision form.

The mixed form (``DeviceRun.set_precision(True, schedule)``) solves each
field equation by defect correction: FP64 residual, FP32 multigrid on the
correction, FP64 accumulation. How much FP32 multigrid work a solve needs
depends on the tree: a deep coarse hierarchy with many base boxes (the 8 mm
Cartesian case has an 8x8-cell coarsest grid) needs more coarse-level cycles
than the two-box axisymmetric tree. The tuner measures that instead of
guessing it.

``tune_schedule`` works in two passes.
  1. Frozen mesh: from a run's current state it advances an FP64 copy
     (bit-identical to the reference's arithmetic) ``n_steps`` steps, and a
     mixed-precision copy per candidate schedule over the same steps. Each
     candidate is timed with CUDA events on its stream (photoionization as
     configured). Its error against the FP64 copy is measured on copies with
     photoionization off, because the photon counts are stochastic: two runs
     draw different photons once a rounded count differs. The errors are:
       - max |E| over the leaf cells, relative;
       - z of the maximum of |E| on the symmetry line (the streamer head),
         relative;
       - max |phi| difference over the leaf cells, relative to max |phi|.
  2. Whole run: in order of increasing step time, each candidate that passed
     pass 1 runs the configuration from its initial conditions to its end
     time, regrids included. Its head position and max |E| are compared with
     the FP64 run's. Errors grow along a run (density errors are integrated
     and amplified by the ionization), so this pass decides.
The first candidate whose errors stay within ``safety`` times the bounds in
both passes is chosen. If none qualifies, the reference's own schedule (FMG,
2/2/base cycles, one correction) is chosen. It tracks the FP64 solve to about
1e-9.
"""
from __future__ import annotations

import itertools
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import metrics
from .device import I_ELEC, I_FLD, I_PHI, clone_state

Schedule = Tuple[int, int, int, int, int]  # fmg, n_cycle_down, n_cycle_up, n_cycle_base, n_corr


def default_candidates(n_cycle_base: int) -> List[Schedule]:
    """Single V-cycles and FMG cycles over a range of smoothing and coarse
    cycles, with one or two correction passes."""
    out: List[Schedule] = []
    bases = sorted({2, 4, 8, 16, 32, n_cycle_base})
    for fmg, ncyc, base, corr in itertools.product((0,), (1, 2), bases, (1, 2)):
        out.append((fmg, ncyc, ncyc, base, corr))
    out.append((1, 1, 1, n_cycle_base, 1))
    out.append((1, 2, 2, n_cycle_base, 1))
    return out


def leaf_ids(levels) -> List[int]:
    return [int(i) for _, (_, lv, _) in sorted(levels.items()) for i in lv]


def leaf_max_abs_diff(x: np.ndarray, y: np.ndarray, meta: np.ndarray, leaves: Sequence[int]) -> float:
    d = 0.0
    for bid in leaves:
        n = int(meta[bid, 14])
        g = n + 2
        a = x[bid, :g * g].reshape(g, g)[1:n + 1, 1:n + 1]
        b = y[bid, :g * g].reshape(g, g)[1:n + 1, 1:n + 1]
        d = max(d, float(np.abs(a - b).max()))
    return d


def errors_against(ref, run, meta, geom, levels, cfg) -> Dict[str, float]:
    """Errors of ``run`` against ``ref`` (two DeviceRuns on the same tree)."""
    leaves = leaf_ids(levels)
    fa, fb = ref.cc(I_FLD), run.cc(I_FLD)
    pa, pb = ref.cc(I_PHI), run.cc(I_PHI)
    ea, eb = ref.cc(I_ELEC), run.cc(I_ELEC)
    za, _, ma = metrics.head_observables(fa, meta, geom, levels, cfg)
    zb, _, mb = metrics.head_observables(fb, meta, geom, levels, cfg)
    pmax = max(leaf_max_abs_diff(pa, np.zeros_like(pa), meta, leaves), 1e-300)
    emax = max(leaf_max_abs_diff(ea, np.zeros_like(ea), meta, leaves), 1e-300)
    return {
        "max_E_rel": abs(ma - mb) / ma,
        "head_z_rel": abs(za - zb) / abs(za),
        "phi_rel": leaf_max_abs_diff(pa, pb, meta, leaves) / pmax,
        "n_e_rel": leaf_max_abs_diff(ea, eb, meta, leaves) / emax,
        "head_z_m": zb,
        "max_E": mb,
    }


def whole_run_observables(cfg, schedule=None):
    """(head z, max |E| on the line, max |E|) of ``cfg`` run from its initial
    conditions to its end time by the driver, FP64 or mixed with
    ``schedule``."""
    from .streamer import Simulation
    sim = Simulation(cfg)
    try:
        if schedule is not None:
            sim.device.set_precision(True, schedule)
        sim.init()
        sim.run(cfg.end_time)
        meta, geom, levels = sim.tree.export()
        return metrics.head_observables(sim.device.cc(I_FLD), meta, geom, levels, cfg)
    finally:
        sim.close()


def time_steps(run, dt: float, n: int) -> float:
    """Mean device time (ms) of n steps of ``run`` on its own stream."""
    import torch
    st = torch.cuda.ExternalStream(run.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st):
        e0.record(st)
        for _ in range(n):
            run.step(dt)
        e1.record(st)
    run.sync()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / n


def tune_schedule(sim, n_steps: int = 200, tol_max_E: float = 1e-4, tol_head_z: float = 5e-3,
                  safety: float = 0.5, candidates: Optional[Sequence[Schedule]] = None,
                  whole_run: bool = True, ref_head=None, n_time: int = 20) -> Dict:
    """Pick the mixed-precision multigrid schedule for ``sim``'s tree and
    configuration (see the module docstring): errors on the frozen mesh after
    ``n_steps`` steps, step time over ``n_time`` steps. ref_head: the FP64
    whole-run observables if the caller has them (else they are computed).
    Returns the choice, its step time and errors, the FP64 step time and the
    table of candidates."""
    import dataclasses
    cfg = sim.cfg
    cfg_np = dataclasses.replace(cfg, photoi_enabled=False) if cfg.photoi_enabled else cfg
    meta, geom, levels = sim.tree.export()
    dt = sim.device.get_max_dt()
    if candidates is None:
        candidates = default_candidates(cfg.n_cycle_base)
    ok_b = lambda e: e["max_E_rel"] <= safety * tol_max_E and e["head_z_rel"] <= safety * tol_head_z
    ref = clone_state(sim)
    ref.step(dt)
    t_fp64 = time_steps(ref, dt, max(1, n_time - 1))
    ref.close()
    ref = clone_state(sim, cfg=cfg_np)
    for _ in range(n_steps):
        ref.step(dt)
    table = []
    for sched in candidates:
        run = clone_state(sim, mixed=True, schedule=sched)
        run.step(dt)
        ms = time_steps(run, dt, max(1, n_time - 1))
        run.close()
        run = clone_state(sim, mixed=True, schedule=sched, cfg=cfg_np)
        for _ in range(n_steps):
            run.step(dt)
        err = errors_against(ref, run, meta, geom, levels, cfg)
        run.close()
        table.append({"schedule": list(sched), "ms": ms, "ok": ok_b(err), **err})
    ref.close()
    if whole_run:
        if ref_head is None:
            ref_head = whole_run_observables(cfg)
        for row in sorted(table, key=lambda r: r["ms"]):
            if not row["ok"]:
                continue
            h = whole_run_observables(cfg, tuple(row["schedule"]))
            row["run_head_z_rel"] = abs(h[0] - ref_head[0]) / abs(ref_head[0])
            row["run_max_E_rel"] = abs(h[2] - ref_head[2]) / ref_head[2]
            row["ok"] = ok_b({"max_E_rel": row["run_max_E_rel"], "head_z_rel": row["run_head_z_rel"]})
            if row["ok"]:
                break
        for row in table:
            if "run_max_E_rel" not in row:
                row["ok"] = False  # not confirmed over a whole run
    good = [r for r in table if r["ok"]]
    if good:
        best = min(good, key=lambda r: r["ms"])
    else:
        fallback = [1, 2, 2, cfg.n_cycle_base, 1]
        best = next((r for r in table if r["schedule"] == fallback), table[-1])
    keys = ("max_E_rel", "head_z_rel", "phi_rel", "n_e_rel", "run_max_E_rel", "run_head_z_rel")
    return {"schedule": tuple(best["schedule"]), "ms": best["ms"], "fp64_ms": t_fp64,
            "speedup": t_fp64 / best["ms"], "errors": {k: best[k] for k in keys if k in best},
            "n_steps": n_steps, "dt": dt, "bounds": {"max_E_rel": tol_max_E, "head_z_rel": tol_head_z,
                                                      "safety": safety},
            "table": table}


def cta_mapping(cells: Sequence[int], total: int, power: float) -> List[int]:
    """Blocks per run of a batch (the box-to-block mapping): one each, and
    the remaining total - n blocks dealt in proportion to cells**power by
    largest remainders (power 0: evenly; 1: in proportion to the tree
    size). Never more than total blocks in all."""
    n = len(cells)
    out = [1] * n
    spare = total - n
    if spare <= 0 or power is None:
        return out
    w = np.asarray([float(c) ** power for c in cells])
    share = spare * w / w.sum()
    base = np.floor(share).astype(int)
    rest = spare - int(base.sum())
    order = np.argsort(-(share - base), kind="stable")
    base[order[:rest]] += 1
    return [1 + int(b) for b in base]


def apply_mapping(sims, total: int, power) -> List[int]:
    """Set each simulation's blocks per launch from its current leaf cells."""
    if power is None:
        return [1] * len(sims)
    m = cta_mapping([s.device.n_leaf_cells() for s in sims], total, power)
    for s, k in zip(sims, m):
        s.device.set_ctas(k)
    return m


def batch_observables(cfgs, schedule=None, use_graph: bool = True, n_threads: int = 8,
                      groups: int = 1, mapping=None, max_blocks: int = 1 << 30):
    """Run ``cfgs`` from their initial conditions to their end times (or
    ``max_blocks`` blocks) as one device-driven batch (FP64, or mixed with
    ``schedule``; ``groups`` pipelined batches). ``mapping``: None for one
    block per run, else (total blocks, power) of ``cta_mapping`` applied to
    the initial trees. Returns the per-run head observables, the batch
    counters (blocks, device ms, host ms, cell updates) and the wall time (s)
    of the batched run."""
    from .streamer import Simulation, run_batch
    sims = [Simulation(c) for c in cfgs]
    try:
        for s in sims:
            if schedule is not None:
                s.device.set_precision(True, schedule)
            s.init()
        if mapping is not None:
            apply_mapping(sims, mapping[0], mapping[1])
        import time
        t0 = time.perf_counter()
        counters = run_batch(sims, [c.end_time for c in cfgs], use_graph=use_graph,
                             n_threads=n_threads, groups=groups, max_blocks=max_blocks)
        wall = time.perf_counter() - t0
        heads = []
        for s, c in zip(sims, cfgs):
            meta, geom, levels = s.tree.export()
            heads.append(metrics.head_observables(s.device.cc(I_FLD), meta, geom, levels, c))
        return heads, counters, wall
    finally:
        for s in sims:
            s.close()


def tune_batch_schedule(cfgs, candidates: Sequence[Schedule], tol_max_E: float = 1e-4,
                        tol_head_z: float = 5e-3, n_threads: int = 8) -> Dict:
    """Schedule of the mixed form for a batch of independent runs. The runs
    are compared with photoionization off (the photon counts are stochastic,
    so two runs with it on drift apart by Monte Carlo noise whatever the
    precision): the FP64 batch once, then each candidate in the given order
    (cheapest first) until every run's head position and max |E| at its end
    time are within the bounds. Returns the choice and per-run errors; if no
    candidate qualifies, the last one."""
    import dataclasses
    quiet = [dataclasses.replace(c, photoi_enabled=False) for c in cfgs]
    ref, _, _ = batch_observables(quiet, None, n_threads=n_threads)
    tried = []
    for sched in candidates:
        heads, _, _ = batch_observables(quiet, tuple(sched), n_threads=n_threads)
        zr = [abs(a[0] - b[0]) / abs(a[0]) for a, b in zip(ref, heads)]
        er = [abs(a[2] - b[2]) / a[2] for a, b in zip(ref, heads)]
        ok = max(zr) <= tol_head_z and max(er) <= tol_max_E
        tried.append({"schedule": list(sched), "head_z_rel_max": max(zr), "max_E_rel_max": max(er),
                      "max_E_rel_median": float(np.median(er)), "ok": ok})
        if ok:
            break
    return {"schedule": tuple(tried[-1]["schedule"]), "errors": tried[-1], "tried": tried,
            "bounds": {"max_E_rel": tol_max_E, "head_z_rel": tol_head_z}}


def tune_batch_mapping(cfgs, schedule=None, total: int = 148,
                       powers: Sequence[Optional[float]] = (None, 0.0, 0.5, 1.0),
                       n_blocks: int = 4, n_threads: int = 8) -> Dict:
    """The box-to-block mapping of a batch, chosen by measurement: for each
    candidate (None: one block per run; else cta_mapping's power) the first
    ``n_blocks`` blocks of the batched run from the initial conditions are
    timed on the device, and the candidate with the highest leaf-cell
    updates per device second wins. The mapping changes only which threads
    do which work, so every candidate gives the same results."""
    table = []
    for pw in powers:
        _, (nb, gpu_ms, _, cu), _ = batch_observables(
            cfgs, schedule, n_threads=n_threads, mapping=None if pw is None else (total, pw),
            max_blocks=n_blocks)
        table.append({"power": pw, "blocks": nb, "device_ms": gpu_ms,
                      "value": cu / (gpu_ms / 1e3) if gpu_ms > 0 else 0.0})
    best = max(table, key=lambda r: r["value"])
    return {"power": best["power"], "total": total, "table": table}
