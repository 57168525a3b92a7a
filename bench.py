#!/usr/bin/env python
"""Benchmark: leaf-cell updates per second per full streamer time step.

One "step" is one full time step of the streamer model on the current mesh
(save old densities, two forward-Euler stages with a field solve after the
first, trapezoidal average, second field solve), i.e. one iteration of the
inner loop of src/streamer_cyl.f90:95-130 (src/streamer_2d.f90:93-128),
including the Monte Carlo photoionization of the step where the workload has
it. The default workload is the axisymmetric 16 mm FP64 case with
photoionization (1e5 photons per step) evolved from its initial conditions
to its end time t = 10 ns with the full regrid cycle; the mesh is then
frozen and K steps are timed at the step size get_max_dt gives. The 8 mm
Cartesian case (t = 2 ns, no photoionization) is --workload cartesian_8mm.

Arms:
  --impl b200       (default) the sm_100a device path through its C ABI
  --impl reference  the CPU implementation of the same path (the oracle port
                    of the reference's Fortran) on all host cores

Multi-GPU (torchrun): one independent replica of the run per rank ("weak"
scaling, no data-path collective); the device time is the max over ranks.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("cell-updates/s per full step, mixed vs FP64 on 1 B200 at stated error; %HBM roof")
UNIT = "cell-updates/s"
# Horizon of the mixed form's frozen-mesh error contract (steps), fixed
# whatever --steps is: errors grow along a run, so a shorter horizon would be
# a weaker contract.
ERR_STEPS = 200
L2_NOTE = "flushed before every timed step (256 MiB write)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["cylindrical_16mm_photoi", "cylindrical_16mm", "cartesian_8mm"],
                    default="cylindrical_16mm_photoi")
    ap.add_argument("--batch", type=int, default=148, help="replicas in the batched extra (0: skip)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision form")
    ap.add_argument("--mixed-schedule", default=None,
                    help="fmg,down,up,base,corr: use this schedule instead of the autotuners' choice")
    ap.add_argument("--runs", type=int, default=64,
                    help="independent uneven runs of the device-driven batch (0: skip)")
    ap.add_argument("--large-level", type=int, default=7,
                    help="uniform level of the large-tree grid-mode extra (7: 4.2M leaf cells, the peak "
                         "size the axisymmetric case's description states; 6: 1M; 0: skip)")
    ap.add_argument("--large-steps", type=int, default=10, help="timed steps of the large-tree extra")
    ap.add_argument("--cube-level", type=int, default=6,
                    help="uniform level of the 3D octree extra (6: 16.8M leaf cells; 0: skip)")
    ap.add_argument("--cube-steps", type=int, default=10, help="timed steps of the 3D extra")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiation extra")
    return ap.parse_args()


def workload_cfg(name):
    from a5_streamer_b200 import config
    if name == "cartesian_8mm":
        return config.cartesian_8mm(), "cartesian_8mm_fp64_t2ns"
    if name == "cylindrical_16mm":
        return config.cylindrical_16mm(), "cylindrical_16mm_fp64_t10ns_no_photoionization"
    return config.cylindrical_16mm(photoi=True), "cylindrical_16mm_photoi_fp64_t10ns"


# ---------------------------------------------------------------------------
class ClockSampler:
    """Samples SM clocks and clock-event reasons through NVML while running."""

    REASONS = {
        "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
        "sw_power_cap": 0x4,
    }

    def __init__(self, index: int, period: float = 0.01):
        self.index, self.period = index, period
        self.samples, self.reasons = [], set()
        self._stop = threading.Event()
        self.max_mhz = None
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                try:
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except Exception:
                    r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                for name, bit in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": len(self.samples)}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_launch(workload):
    """DRAM bytes per step launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"a5g_step_{workload}.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["dram_bytes_per_launch"])
    except Exception:
        return None


# ---------------------------------------------------------------------------
def cpu_baseline(cfg, seconds, threads):
    """The oracle port of the reference's algorithm on the host cores: the same
    run to the end time, then as many full steps as fit in the budget."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import a5ref
    sim = a5ref.Sim(cfg, n_threads=threads)
    sim.init()
    sim.run(cfg.end_time)
    n_leaf = sim.n_leaf_cells()
    dt = sim.get_max_dt()
    sim.step(dt)  # warm
    steps, t0 = 0, time.perf_counter()
    while True:
        sim.step(dt)
        steps += 1
        el = time.perf_counter() - t0
        if el > seconds or steps >= 100000:
            break
    return n_leaf * steps / el, steps, el, n_leaf


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cfg, wname = workload_cfg(args.workload)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import a5ref
    import numpy as np
    threads = os.cpu_count() or 1
    world = int(os.environ.get("WORLD_SIZE", "1"))
    sim = a5ref.Sim(cfg, n_threads=threads)
    sim.init()
    sim.run(cfg.end_time)
    n_leaf = sim.n_leaf_cells()
    dt = sim.get_max_dt()
    for _ in range(args.warmup):
        sim.step(dt)
    photons = sim.photons_created() if cfg.photoi_enabled else 0
    # the device arm's protocol: a 256 MiB write before every timed step
    # (outside the timed region), here to the host caches
    flush = np.zeros(256 << 20, dtype=np.uint8)
    el = 0.0
    for k in range(args.steps):
        flush.fill(k & 0xFF)
        t0 = time.perf_counter()
        sim.step(dt)
        el += time.perf_counter() - t0
    value = n_leaf * args.steps / el
    meta = sim.meta()
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wname, "leaf_cells": n_leaf, "boxes_in_use": int(meta[:, 0].sum()),
                   "min_lvl": sim.min_lvl, "max_lvl": sim.max_lvl,
                   "precision": "fp64", "parallelism": f"replicas{world}",
                   "photons_per_step": photons, "l2": L2_NOTE},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full steps of the {wname} mesh at t_end, "
                                   f"OpenMP over the boxes of each level"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_uneven_batch(n_runs, first_schedule, fixed=False):
    """The batched form: n independent axisymmetric runs of uneven size
    (config.batch_cylindrical_runs: seeded background density, field, domain
    length; photoionization on) from their initial conditions to their own
    end time (5 ns), stepped together by the device-driven batch (one launch
    per kernel per step for all runs, each block replayed from a CUDA graph,
    regrids on host threads). The mixed form's schedule comes from the batch
    tuner (whole-run errors of every run against FP64, photoionization off);
    throughput is measured with photoionization on, in FP64 and mixed."""
    from a5_streamer_b200 import autotune, config
    cfgs = config.batch_cylindrical_runs(n_runs)
    threads = os.cpu_count() or 1
    cands = [tuple(first_schedule)] + [c for c in [(0, 2, 2, 4, 1), (0, 2, 2, 4, 2), (1, 1, 1, 4, 1),
                                                    (1, 2, 2, 4, 1)] if c != tuple(first_schedule)]
    if fixed:
        tuned = {"schedule": tuple(first_schedule), "errors": None, "tried": []}
    else:
        tuned = autotune.tune_batch_schedule(cfgs, cands, n_threads=threads)
    sched = tuned["schedule"]
    out = {"runs": n_runs, "generator": "numpy default_rng(20261203)", "t_end": cfgs[0].end_time,
           "domain_z_mm": [min(c.domain_len[1] for c in cfgs) * 1e3, max(c.domain_len[1] for c in cfgs) * 1e3],
           "photoionization": True}
    heads = {}
    import torch
    from a5_streamer_b200 import device as dv
    probe = dv.DeviceRun(cfgs[0])
    total = probe.ctas()[1]
    probe.close()
    for form, sc in (("fp64", None), ("mixed", sched)):
        # box-to-block mapping of this form, by measurement (a few blocks)
        tm = autotune.tune_batch_mapping(cfgs, sc, total=total, n_threads=threads)
        mapping = None if tm["power"] is None else (total, tm["power"])
        # one batch: the blocks' device time; two pipelined groups: the wall
        # time of the whole batched run with the host regrids overlapped
        # the wall time includes the host regrids, which share the host with
        # other work: the faster of two whole batched runs is reported
        best = None
        for rep in range(2):
            if rep == 0:
                torch.cuda.nvtx.range_push(f"uneven_{form}")  # profilers select the first run
            res = autotune.batch_observables(cfgs, sc, n_threads=threads, mapping=mapping)
            if rep == 0:
                torch.cuda.nvtx.range_pop()
            if best is None or res[2] < best[2]:
                best = res
        h, (nb, gpu_ms, host_ms, cu), wall1 = best
        _, (_, _, host2, cu2), wall2 = autotune.batch_observables(cfgs, sc, n_threads=threads, groups=2,
                                                                   mapping=mapping)
        heads[form] = h
        out[form] = {"value": cu / (gpu_ms / 1e3), "unit": UNIT, "device_s": gpu_ms / 1e3,
                     "host_regrid_s": host_ms / 1e3, "blocks": nb, "cell_updates": cu,
                     "value_wall": cu / wall1, "wall_s": wall1, "wall_of": "faster of 2 batched runs",
                     "value_wall_two_groups": cu2 / wall2, "wall_s_two_groups": wall2,
                     "mapping": {"chosen_power": tm["power"], "blocks": total, "tuner": tm["table"],
                                 "note": "power None: one block per run; p: one each plus the rest "
                                         "in proportion to leaf cells^p"}}
    er = [abs(a[2] - b[2]) / a[2] for a, b in zip(heads["fp64"], heads["mixed"])]
    out["mixed"]["schedule"] = list(sched)
    out["mixed"]["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["mixed"]["errors_vs_fp64_photoionization_off"] = tuned["errors"]
    out["mixed"]["tuner_tried"] = tuned["tried"]
    out["mixed"]["max_E_rel_photoionization_on"] = {
        "max": max(er), "median": statistics.median(er),
        "note": "photon counts are stochastic: two runs draw different photons once a rounded count differs"}
    return out


def run_uneven_sharded(n_runs, schedule, rank, world, device="cuda"):
    """The uneven batch over `world` ranks: the runs dealt by estimated cost
    (domain area, proportional to the leaf cells of the initial mesh) with
    replicas.partition_runs, each rank stepping its share by the
    device-driven batch with no data-path collective; the schedule of the
    mixed form is the single-run tuner's, not re-tuned. Whole-job value:
    cell updates summed over ranks / the slowest rank's device time. Every
    rank makes the same reductions in the same order after its local work,
    also when that work failed."""
    from a5_streamer_b200 import autotune, config, replicas
    cfgs = config.batch_cylindrical_runs(n_runs)
    mine = replicas.partition_runs([c.domain_len[0] * c.domain_len[1] for c in cfgs], world)[rank]
    threads = max(1, (os.cpu_count() or 1) // world)
    out = {"runs": n_runs, "ranks": world, "runs_per_rank": len(mine), "generator": "numpy default_rng(20261203)",
           "t_end": cfgs[0].end_time, "partition": "replicas.partition_runs by domain area (LPT)",
           "schedule_mixed": list(schedule)}
    for form, sc in (("fp64", None), ("mixed", tuple(schedule))):
        ok, dev_s, cu, wall = 1.0, 0.0, 0.0, 0.0
        err = ""
        try:
            if mine:
                _, (_, gpu_ms, _, cu), wall = autotune.batch_observables([cfgs[i] for i in mine], sc,
                                                                          n_threads=threads)
                dev_s = gpu_ms / 1e3
        except Exception as exc:  # reported after the reductions, which every rank makes
            ok, err = 0.0, str(exc)
        ok_all = -replicas.max_over_ranks(-ok, device=device)
        dev_max = replicas.max_over_ranks(dev_s, device=device)
        cu_sum = replicas.sum_over_ranks(cu, device=device)
        wall_max = replicas.max_over_ranks(wall, device=device)
        if ok_all < 1.0:
            out[form] = {"unavailable": err or "failed on another rank"}
        else:
            out[form] = {"value": cu_sum / dev_max, "unit": UNIT, "device_s_max_over_ranks": dev_max,
                         "cell_updates": cu_sum, "value_wall": cu_sum / wall_max, "wall_s_max_over_ranks": wall_max}
    if "value" in out["fp64"] and "value" in out["mixed"]:
        out["mixed"]["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def run_large_tree(level, steps, warmup, flush, clock_index):
    """The grid-mode form on a large tree: the 8 mm Cartesian case on a
    uniformly refined mesh of the given level (config.cartesian_uniform;
    level 6: 1,048,576 leaf cells), one run on all co-resident blocks of the
    GPU (a5g_set_ctas), FP64 and mixed; for comparison the same steps on one
    block. Steps on the initial mesh at the step size get_max_dt gives, L2
    flushed before each, CUDA events on the run's stream."""
    import torch
    from a5_streamer_b200 import config, metrics, streamer
    cfg = config.cartesian_uniform(level)
    sim = streamer.Simulation(cfg)
    run = sim.device
    n_cta = run.ctas()[1]
    run.set_ctas(n_cta)
    sim.init()
    n_leaf = run.n_leaf_cells()
    meta, _, levels = sim.tree.export()
    cen = metrics.census(meta, levels, cfg.box_size)
    bytes_step = metrics.bytes_per_step(cen)
    dt = run.get_max_dt()
    st = torch.cuda.ExternalStream(run.stream_ptr())

    def timed(n):
        for _ in range(warmup):
            run.step(dt)
        run.sync()
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(n)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(n)]
        with torch.cuda.stream(st):
            for k in range(n):
                flush.fill_(k & 0xFF)
                e0[k].record(st)
                run.step(dt)
                e1[k].record(st)
        run.sync()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in zip(e0, e1)) / n

    with ClockSampler(clock_index) as clk:
        torch.cuda.nvtx.range_push("large_tree_grid")
        ms = timed(steps)
        torch.cuda.nvtx.range_pop()
    peak = measured_peak()[0]
    gbs = bytes_step / (ms / 1e3) / 1e9
    out = {"workload": f"cartesian_uniform_lvl{level}", "leaf_cells": n_leaf,
           "boxes_in_use": int(meta[:, 0].sum()), "min_lvl": sim.tree.min_lvl, "max_lvl": sim.tree.max_lvl,
           "n_cta": n_cta, "ms_per_step": ms, "value": n_leaf / (ms / 1e3), "unit": UNIT,
           "algorithmic_bytes_per_step": bytes_step, "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / peak,
           "clocks": clk.summary()}
    # the mixed form on the same blocks (the reference's FMG schedule for
    # the FP32 correction solve, which tracks FP64 to ~1e-9)
    run.set_precision(True, (1, 2, 2, cfg.n_cycle_base, 1))
    ms_m = timed(steps)
    run.set_precision(False)
    out["mixed"] = {"ms_per_step": ms_m, "value": n_leaf / (ms_m / 1e3),
                    "speedup_vs_fp64": ms / ms_m, "schedule": [1, 2, 2, cfg.n_cycle_base, 1]}
    # one block, as the small trees run
    run.set_ctas(1)
    ms1 = timed(max(2, steps // 5))
    out["one_block"] = {"ms_per_step": ms1, "value": n_leaf / (ms1 / 1e3),
                        "grid_speedup": ms1 / ms}
    sim.close()
    return out


def run_cube_3d(level, steps, warmup, flush, clock_index, cpu_seconds=3.0):
    """The 3D octree form (include/a5g3.h): the 16 mm cube of the 3D case on a
    uniformly refined octree of the given level (6: 16,777,216 leaf cells,
    dx = 62.5 um), FP64, initial conditions and first field solve on the
    device, then steps at the step size get_max_dt gives, each a replay of the
    captured step graph, L2 flushed before each, CUDA events on the run's
    stream. Beside it, the oracle's 3D step on a level-4 cube (262,144 leaf
    cells) timed on the host cores for about cpu_seconds."""
    import torch
    from a5_streamer_b200 import config, device3
    cfg = config.cube_16mm_uniform(level)
    run = device3.Run3(cfg)
    run.init()
    run.sync()
    dt = run.get_max_dt()
    st = torch.cuda.ExternalStream(run.stream_ptr())
    for _ in range(warmup):
        run.step(dt)
    run.sync()
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    with ClockSampler(clock_index) as clk:
        torch.cuda.nvtx.range_push("octree_3d")
        with torch.cuda.stream(st):
            for k in range(steps):
                flush.fill_(k & 0xFF)
                e0[k].record(st)
                run.step(dt)
                e1[k].record(st)
        run.sync()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = sum(a.elapsed_time(b) for a, b in zip(e0, e1)) / steps
    bytes_step = run.bytes_per_step()
    peak = measured_peak()[0]
    gbs = bytes_step / (ms / 1e3) / 1e9
    n_leaf = run.n_leaf_cells
    out = {"workload": f"cube_16mm_uniform_lvl{level}", "leaf_cells": n_leaf, "boxes": run.max_id,
           "min_lvl": run.min_lvl, "max_lvl": run.max_lvl, "precision": "fp64",
           "ms_per_step": ms, "value": n_leaf / (ms / 1e3), "unit": UNIT,
           "algorithmic_bytes_per_step": bytes_step, "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / peak,
           "clocks": clk.summary(), "l2": L2_NOTE}
    # the mixed form from the same initial state, the same steps; errors of
    # its end state against the FP64 run's
    E64, z64 = head_3d(run)
    out["mixed"] = {}
    for name, sched in (("reference_schedule", None), ("vcycle_2corr", (0, 1, 1, 4, 2))):
        mx = device3.Run3(cfg)
        mx.init()
        mx.set_precision(True, sched)
        mx.sync()
        for _ in range(warmup):
            mx.step(dt)
        mx.sync()
        stm = torch.cuda.ExternalStream(mx.stream_ptr())
        f0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        f1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        with ClockSampler(clock_index) as clk2:
            torch.cuda.nvtx.range_push("octree_3d_mixed_" + name)
            with torch.cuda.stream(stm):
                for k in range(steps):
                    flush.fill_(k & 0xFF)
                    f0[k].record(stm)
                    mx.step(dt)
                    f1[k].record(stm)
            mx.sync()
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
        ms_m = sum(a.elapsed_time(b) for a, b in zip(f0, f1)) / steps
        Em, zm = head_3d(mx)
        out["mixed"][name] = {
            "schedule": list(sched) if sched else [1, 2, 2, cfg.n_cycle_base, 1],
            "ms_per_step": ms_m, "value": n_leaf / (ms_m / 1e3), "speedup_vs_fp64": ms / ms_m,
            "errors_vs_fp64": {"steps": warmup + steps, "max_E_rel": abs(Em - E64) / E64,
                               "head_z_rel": abs(zm - z64) / z64},
            "clocks": clk2.summary()}
        mx.close()
    out["mixed"]["bounds"] = {"max_E_rel": 1e-4, "head_z_rel": 5e-3}
    run.close()
    # the oracle's 3D step on the host cores (a bounded sample on a smaller cube)
    try:
        if cpu_seconds <= 0:
            raise RuntimeError("skipped (--no-cpu-baseline)")
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import a5ref
        cfg4 = config.cube_16mm_uniform(4)
        sim = a5ref.Sim3(cfg4, n_threads=os.cpu_count() or 1)
        sim.init()
        dt4 = sim.get_max_dt()
        t0, n = time.perf_counter(), 0
        while time.perf_counter() - t0 < cpu_seconds:
            sim.step(dt4)
            n += 1
        el = time.perf_counter() - t0
        out["cpu_port"] = {"value": sim.n_leaf_cells() * n / el, "unit": UNIT, "cores": os.cpu_count() or 1,
                           "sample": f"{n} steps ({el:.1f} s) of the level-4 cube (262,144 leaf cells), "
                                     "oracle port, OpenMP over the boxes of each level"}
        sim.close()
    except Exception as exc:  # the oracle is test infrastructure; report, do not fail
        out["cpu_port"] = {"unavailable": str(exc)}
    return out


def run_adjoint(reps=3):
    """The differentiation addition (include/a5a.h): the 8 mm Cartesian case
    without photoionization, 200 steps at the nominal step-size schedule on
    the mesh of the initial refinement, checkpoints every 20 steps; the head
    observable's gradient with respect to (mu, D, A, B, E_bg). Timed (wall
    clock, each call synchronised): the program alone (a5a_forward) and the
    gradient (a5a_gradient: forward pass with stored states, recomputation of
    each interval, reverse pass); errors of the gradient against central
    differences (h = 1e-6 relative) of the device program."""
    import numpy as np
    from a5_streamer_b200 import adjoint, streamer
    prob = adjoint.HeadProblem()
    cfg = prob.config()
    sim = streamer.Simulation(cfg)
    sim.init()
    adj = adjoint.HeadAdjoint(sim, prob)
    dts, T = adj.schedule()
    adj.bind()
    p0 = prob.nominal()
    adj.value(p0)
    adj.gradient(p0)
    tf, tg = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        J = adj.value(p0)
        tf.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        J2, g = adj.gradient(p0)
        tg.append(time.perf_counter() - t0)
    fd = np.zeros(5)
    for k in range(5):
        v = []
        for sg in (1.0, -1.0):
            p = p0.copy()
            p[k] *= 1 + sg * 1e-6
            v.append(adj.value(p))
        fd[k] = (v[0] - v[1]) / (2e-6 * p0[k])
    adj.close()
    n_leaf = sim.device.n_leaf_cells()
    sim.close()
    rel = np.abs(g - fd) / np.abs(fd)
    return {"workload": "cartesian_8mm fixed mesh, 200 steps, checkpoints every 20, photoionization off",
            "leaf_cells": n_leaf, "steps": prob.n_steps, "observable": "head height at x = 4 mm",
            "temperature_V_per_m": T, "tau_m": prob.tau, "J_m": J,
            "params": list(adjoint.PARAM_NAMES), "p0": p0.tolist(),
            "dJ_dp": g.tolist(), "dJ_dlnp": (g * p0).tolist(), "fd": fd.tolist(),
            "rel_err_vs_fd": rel.tolist(), "max_rel_err_vs_fd": float(rel.max()),
            "forward_s": min(tf), "gradient_s": min(tg), "gradient_over_forward": min(tg) / min(tf),
            "timing": f"wall clock, best of {reps}, each call synchronised"}


def head_3d(run):
    """(max |E| over the leaves, height of the cell holding it) of a 3D run."""
    import numpy as np
    E = run.cc(5)
    meta = run.meta()
    lvl, g = run.max_lvl, run.nc + 2
    ids = run.levels()[lvl][0]
    sub = E[ids].reshape(len(ids), g, g, g)[:, 1:-1, 1:-1, 1:-1]
    q = np.unravel_index(np.argmax(sub), sub.shape)
    dr = run.cfg.dr_at(lvl)
    z = (meta[ids[q[0]], 4] - 1) * run.nc * dr + (q[1] + 0.5) * dr
    return float(sub[q]), float(z)


def moving_streamer_errors(schedule):
    """Errors of the mixed form where the streamer moves: the 8 mm Cartesian
    case at E_bg = 7 MV/m (levels up to 6, no photoionization), whose head
    travels from z = 7 mm to about 3.5 mm by its end time (2 ns). The tuner
    picks the schedule for this tree (200-step frozen-mesh errors from the
    state at 1 ns, then whole runs); its head position (argmax of |E| on the
    symmetry line) and max |E| at the end time are compared with the FP64
    run, and its step time with FP64's. The schedule tuned for the benchmark's
    axisymmetric tree is run here too: a schedule does not transfer between
    trees (this one's coarsest grid is 8x8 cells), which is why the tuner
    works per tree. In the benchmark's own cases the head stays in one cell,
    so their head error is 0 by construction."""
    from a5_streamer_b200 import autotune, config, streamer
    cfg = config.cartesian_8mm(applied_fld=7e6, lvls_max=6)
    h64 = autotune.whole_run_observables(cfg)
    sim = streamer.Simulation(cfg)
    sim.init()
    sim.run(0.5 * cfg.end_time)
    tuned = autotune.tune_schedule(sim, n_steps=ERR_STEPS, ref_head=h64)
    sim.close()
    own = tuple(tuned["schedule"])
    hmx = autotune.whole_run_observables(cfg, own)
    hxf = autotune.whole_run_observables(cfg, tuple(schedule))
    return {"case": "cartesian_8mm E_bg=7MV/m lvls_max=6 t=2ns, photoionization off",
            "head_z_m": {"seed": cfg.seeds[0].r0[1], "fp64": h64[0], "mixed": hmx[0]},
            "schedule": list(own), "head_z_rel": abs(hmx[0] - h64[0]) / abs(h64[0]),
            "max_E_rel": abs(hmx[2] - h64[2]) / h64[2],
            "errors_after_steps": {k: tuned["errors"].get(k) for k in ("max_E_rel", "head_z_rel")},
            "speedup_vs_fp64": tuned["speedup"], "ms_per_step": tuned["ms"], "fp64_ms_per_step": tuned["fp64_ms"],
            "bench_tree_schedule": {"schedule": list(schedule),
                                    "head_z_rel": abs(hxf[0] - h64[0]) / abs(h64[0]),
                                    "max_E_rel": abs(hxf[2] - h64[2]) / h64[2]},
            "bounds": {"max_E_rel": 1e-4, "head_z_rel": 5e-3}}


def run_b200(args):
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from a5_streamer_b200 import build, metrics, replicas, streamer
    from a5_streamer_b200 import device as dv
    build.build()  # no-op when the in-tree library is current

    cfg, wname = workload_cfg(args.workload)
    sim = streamer.Simulation(cfg)
    sim.init()
    sim.run(cfg.end_time)
    run = sim.device
    n_leaf = run.n_leaf_cells()
    meta, geom, levels = sim.tree.export()
    head_fp64 = metrics.head_observables(run.cc(dv.I_FLD), meta, geom, levels, cfg)
    cen = metrics.census(meta, levels, cfg.box_size)
    dt = run.get_max_dt()

    ext = torch.cuda.ExternalStream(run.stream_ptr())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    for _ in range(args.warmup):
        run.step(dt)
    run.sync()
    torch.cuda.synchronize()
    photons = run.photon_stats()[0] if cfg.photoi_enabled else 0
    bytes_step = metrics.bytes_per_step(cen, photons=photons)
    launches_per_step = 3 if cfg.photoi_enabled else 1
    if dist:
        dist.barrier()

    K = args.steps
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    with ClockSampler(local) as clk:
        # NVTX range "timed": lets a profiler select the launches of the timed
        # region (ncu --nvtx --nvtx-include "timed/")
        torch.cuda.nvtx.range_push("timed")
        with torch.cuda.stream(ext):
            for k in range(K):
                flush.fill_(k & 0xFF)
                e0[k].record(ext)
                run.step(dt)
                e1[k].record(ext)
        torch.cuda.nvtx.range_pop()
        run.sync()
        torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in zip(e0, e1)]
    total_s = replicas.max_over_ranks(sum(step_ms) / 1e3, device="cuda")
    value = replicas.replica_throughput(n_leaf * K * world, total_s)
    ms_per_step = 1e3 * total_s / K

    # end to end through the public API: dt computed from device reductions
    # read back to the host each step, the step launched with the host dt
    run.sync()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        d = run.get_max_dt()
        run.step(d)
    run.sync()
    e2e_s = replicas.max_over_ranks(time.perf_counter() - t0, device="cuda")
    e2e = {"value": replicas.replica_throughput(n_leaf * K * world, e2e_s), "unit": UNIT,
           "h2d_bytes_per_step": 8, "d2h_bytes_per_step": 24}

    def time_batch(mixed, schedule=None):
        """B replicas of the same mesh and state, one block each, one launch
        per kernel per step; L2 flushed before every timed step."""
        reps = [dv.clone_state(sim, mixed=mixed, schedule=schedule) for _ in range(args.batch)]
        bstream = torch.cuda.ExternalStream(reps[0].stream_ptr())
        dts = [dt] * len(reps)
        for _ in range(2):
            dv.step_batch(reps, dts)
        reps[0].sync()
        nb = max(3, K // 10)
        b0 = [torch.cuda.Event(enable_timing=True) for _ in range(nb)]
        b1 = [torch.cuda.Event(enable_timing=True) for _ in range(nb)]
        with ClockSampler(local) as bclk:
            torch.cuda.nvtx.range_push("batched_mixed" if mixed else "batched_fp64")
            with torch.cuda.stream(bstream):
                # a head start for the host: the device spins (a fixed number
                # of cycles, about 100 ms) while the host queues the timed
                # steps, so that host work between launches (a stream check
                # per member) cannot leave the device idle inside the events
                torch.cuda._sleep(int(100e-3 * 1.965e9))
                for k in range(nb):
                    flush.fill_(k & 0xFF)
                    b0[k].record(bstream)
                    dv.step_batch(reps, dts)
                    b1[k].record(bstream)
            torch.cuda.nvtx.range_pop()
            reps[0].sync()
            torch.cuda.synchronize()
        bt = sum(a.elapsed_time(b) for a, b in zip(b0, b1)) / 1e3
        for r in reps:
            r.close()
        gbs = bytes_step * len(reps) * nb / bt / 1e9
        return {"replicas": len(reps), "steps": nb, "value": n_leaf * len(reps) * nb / bt,
                "unit": UNIT, "ms_per_step": 1e3 * bt / nb,
                "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / measured_peak()[0],
                "clocks": bclk.summary()}

    def time_single(r, label):
        """K steps of one run, L2 flushed before each, CUDA events on its stream."""
        st = torch.cuda.ExternalStream(r.stream_ptr())
        for _ in range(args.warmup):
            r.step(dt)
        r.sync()
        a0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        a1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        torch.cuda.nvtx.range_push(label)
        with torch.cuda.stream(st):
            for k in range(K):
                flush.fill_(k & 0xFF)
                a0[k].record(st)
                r.step(dt)
                a1[k].record(st)
        torch.cuda.nvtx.range_pop()
        r.sync()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in zip(a0, a1)) / K

    batched = time_batch(False) if args.batch > 0 else None

    # mixed-precision form: schedule picked by the autotuner on this tree,
    # errors against the FP64 path (bit-identical to the reference's
    # arithmetic) over K steps from the same state and over a whole run
    mixed = None
    if not args.no_mixed:
        from a5_streamer_b200 import autotune
        import dataclasses
        if args.mixed_schedule:
            sched = tuple(int(v) for v in args.mixed_schedule.split(","))
            tuned = {"schedule": sched, "table": [], "n_steps": 0}
        else:
            # the frozen-mesh check over the fixed error horizon (ERR_STEPS
            # steps, whatever K is) and the whole run to the end time
            tuned = autotune.tune_schedule(sim, n_steps=ERR_STEPS, ref_head=head_fp64)
            sched = tuned["schedule"]
        mrun = dv.clone_state(sim, mixed=True, schedule=sched)
        m_ms = time_single(mrun, "timed_mixed")
        mrun.close()
        # ERR_STEPS steps on the frozen mesh, photoionization off in both
        # copies (the photon counts are stochastic and would diverge)
        cfg_np = dataclasses.replace(cfg, photoi_enabled=False)
        a = dv.clone_state(sim, cfg=cfg_np)
        b = dv.clone_state(sim, mixed=True, schedule=sched, cfg=cfg_np)
        for _ in range(ERR_STEPS):
            a.step(dt)
            b.step(dt)
        a.sync()
        b.sync()
        err_k = autotune.errors_against(a, b, meta, geom, levels, cfg)
        a.close()
        b.close()
        head_m = autotune.whole_run_observables(cfg, sched)
        mixed = {
            "value": n_leaf / (m_ms / 1e3), "unit": UNIT, "ms_per_step": m_ms,
            "speedup_vs_fp64": ms_per_step / m_ms, "dtype": "f32 fluxes/lookups/smoothing, f64 residual/potential/densities/dt",
            "schedule": {"fmg": sched[0], "n_cycle_down": sched[1], "n_cycle_up": sched[2],
                         "n_cycle_base": sched[3], "n_corr": sched[4]},
            "errors_after_steps": {"steps": ERR_STEPS, "photoionization": False,
                                   **{k: err_k[k] for k in ("max_E_rel", "head_z_rel", "phi_rel", "n_e_rel")}},
            "errors_whole_run": {"t_end": cfg.end_time,
                                 "head_z_rel": abs(head_m[0] - head_fp64[0]) / abs(head_fp64[0]),
                                 "max_E_rel": abs(head_m[2] - head_fp64[2]) / head_fp64[2],
                                 "head_z_m": [head_fp64[0], head_m[0]], "max_E": [head_fp64[2], head_m[2]],
                                 "photoionization": bool(cfg.photoi_enabled),
                                 "note": ("photon counts are stochastic: the two runs draw different photons "
                                          "once a cell's rounded count differs") if cfg.photoi_enabled else ""},
            "bounds": {"max_E_rel": 1e-4, "head_z_rel": 5e-3},
            "tuner": {"candidates": len(tuned["table"]), "frozen_mesh_steps": tuned["n_steps"],
                      "whole_run": True},
            "errors_moving_streamer": moving_streamer_errors(sched),
            "batched": time_batch(True, sched) if args.batch > 0 else None,
        }
        if batched and mixed["batched"]:
            mixed["batched"]["speedup_vs_fp64"] = mixed["batched"]["value"] / batched["value"]

    large = None
    if args.large_level > 0 and rank == 0:
        large = run_large_tree(args.large_level, args.large_steps, 3, flush, local)
    cube = None
    if args.cube_level > 0 and rank == 0:
        cube = run_cube_3d(args.cube_level, args.cube_steps, 3, flush, local,
                           cpu_seconds=0.0 if args.no_cpu_baseline else 3.0)

    adj = None
    if not args.no_adjoint and rank == 0:
        adj = run_adjoint()

    uneven = None
    if args.runs > 0:
        sched_u = mixed["schedule"] if mixed else None
        sched_u = (sched_u["fmg"], sched_u["n_cycle_down"], sched_u["n_cycle_up"], sched_u["n_cycle_base"],
                   sched_u["n_corr"]) if sched_u else (1, 2, 2, cfg.n_cycle_base, 1)
        if world == 1:
            uneven = run_uneven_batch(args.runs, sched_u, fixed=bool(args.mixed_schedule))
        else:
            uneven = run_uneven_sharded(args.runs, sched_u, rank, world)

    peak, peak_kind = measured_peak()
    achieved = bytes_step / (ms_per_step / 1e3) / 1e9
    traffic = traffic_per_launch(args.workload)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "peak_kind": peak_kind, "algorithmic_bytes_per_launch": bytes_step,
                "timed_unit": "one full step" + (" (photon sources, absorption, step kernel)"
                                                 if cfg.photoi_enabled else " (step kernel)")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, steps, el, nl = cpu_baseline(cfg, args.cpu_seconds, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{steps} full steps ({el:.1f} s) of the same mesh at t_end, "
                         f"oracle port, OpenMP over the boxes of each level"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wname, "leaf_cells": n_leaf, "boxes_in_use": int(meta[:, 0].sum()),
                       "min_lvl": sim.tree.min_lvl, "max_lvl": sim.tree.max_lvl,
                       "precision": "fp64", "parallelism": f"replicas{world}",
                       "photons_per_step": photons,
                       "l2": L2_NOTE},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": K * launches_per_step,
            "clocks": clk.summary(), "batched": batched, "mixed": mixed,
            "uneven_batch": uneven, "large_tree": large, "octree_3d": cube,
            "adjoint": adj,
        }
        print(json.dumps(out), flush=True)
    sim.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
