"""Benchmark: compartment-steps/s of the per-micro-step loop on the seeded config-2 network.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]
                    [--cells C] [--precision fp64|mixed|both]

Workload: 10,000 cells with uneven random binary trees (total compartments
uniform in [100, 1000]), 100 Exp2Syn per cell, recurrent NetCons (delays
U[1,5] ms), a 5 Hz Poisson NetStim per synapse, dt = 0.025 ms — the seeded
synthetic network of mind_b200.networks.config2 (no dataset is involved).
A step is one micro step of the whole network.  `value` is whole-job
compartment-steps/s with all state resident in HBM; `e2e` is the same metric
through the public run() call (C-ABI), including the host copies of the
recorded soma voltages and the spike raster.  Under torchrun (N GPUs) the
config-2 network has 10,000 x N cells, each rank owning 10,000 of them (weak
scaling): NetCons from cells on other ranks arrive as external spike inputs,
and the ranks all-gather their cells' spikes over NCCL once per window
(mind_b200.sharding); config 3 runs one network per rank.  Timing is CUDA
events around the window loop, exchanges included, max over ranks.
--impl reference times the CPU FP64 restatement of the
reference's step loop (oracle/) on the host cores; MIND.jl itself is Julia
and cannot run on this box.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mind.jl_b200"))

import numpy as np  # noqa: E402

COLLECTIVE_DEVICE = "cuda"   # device of the tensors handed to torch.distributed
METRIC = "compartment-steps/s (config 2: 10,000 uneven cells, recurrent Exp2Syn, dt 0.025 ms)"
WORKLOAD_METRICS = {
    2: METRIC,
    3: "compartment-steps/s (config 3: 1,000 uneven cells, 3e5 NetStim-driven Exp2Syn, dt 0.025 ms)",
    4: "compartment-steps/s (config 4: 2,000 uneven cells coupled to 20 Jansen-Rit regions, dt 0.025 ms)",
}
UNIT = "compartment-steps/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=800)
    p.add_argument("--warmup", type=int, default=40)
    p.add_argument("--impl", default="mine", choices=["mine", "reference"])
    p.add_argument("--cells", type=int, default=None, help="cells (default: the configuration's count)")
    p.add_argument("--config", type=int, default=2, choices=[2, 3, 4, 5],
                   help="2: 10,000 uneven binary-tree cells (the headline); 3: 1,000 pyramidal-like cells; "
                        "4: 2,000 pyramidal-like cells coupled to 20 Jansen-Rit regions; 5 (with --surrogate): "
                        "100,000 config-4 cells in 200 populations")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep 128 threads per cell in every size bin instead of timing the shapes")
    p.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"],
                   help="both: the FP64 headline plus the mixed mode and its accuracy against FP64")
    p.add_argument("--accuracy-ms", type=float, default=0.0,
                   help="instead of timing: run FP64 and mixed from t=0 for this long and print their differences")
    p.add_argument("--surrogate", action="store_true",
                   help="config 4: train the spike-output surrogate on a detailed run, then time the coupled run "
                        "with 98%% of the cells replaced, against the plain FP64 run, and their region rates")
    p.add_argument("--eval-ms", type=float, default=None,
                   help="--surrogate: simulated time of the evaluation runs (default 1000 ms for config 4, "
                        "100 ms for config 5); longer runs shrink the counting noise of the region rates")
    p.add_argument("--settle-ms", type=float, default=50.0,
                   help="simulated time advanced untimed before --warmup in both arms, so the timed steps run "
                        "on an active network (recurrent cell spikes, routing, NET_RECEIVE); config.t_start_ms")
    p.add_argument("--cpu-steps", type=int, default=8)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def build_network(cells, seed: int, config: int = 2, rank: int = 0, world: int = 1):
    """Config 3 (one network per rank), or rank `rank`'s block of a config-2 network of
    `cells` x `world` cells (world = 1: the whole 10,000-cell network)."""
    import mind_b200 as mb
    from mind_b200 import networks

    if config == 5:
        model = networks.config5(n_cells=cells or 100_000)
    elif config == 4:
        model = networks.config4(n_cells=cells or 2000)
    elif config == 3:
        model = networks.config3(n_cells=cells or 1000)
    else:
        model = networks.config2(n_cells=cells or 10000, rank=rank, world=world)
    layout = mb.build(model, seed=seed)
    return model, layout


def algorithmic_bytes_per_step(layout, events_per_step: float) -> float:
    """Minimal one-pass HBM traffic of one FP64 micro step.

    Per node 44 B (v read+write, parent index, axial, C, axial_diagonal); per
    pas row 24 B; per hh row 104 B; per Exp2Syn row 68 B; per ExpSyn row 36 B;
    per delivered event 44 B.
    """
    per_kind = {"pas": 24, "hh": 104, "Exp2Syn": 68, "ExpSyn": 36, "IClamp": 28}
    total = 44.0 * layout.n_nodes
    for g in layout.groups:
        total += per_kind.get(g.mechanism.name, 0) * g.rows
    return total + 44.0 * events_per_step


def delivered_events(layout, spike_sids) -> int:
    if len(spike_sids) == 0:
        return 0
    index = {int(s): k for k, s in enumerate(layout.source_ids)}
    fan = np.diff(layout.fanout_offsets)
    return int(sum(fan[index[int(s)]] for s in spike_sids))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        self.file.seek(0)
        rows = [r.strip().split(", ") for r in self.file.read().splitlines() if r.strip()]
        sm, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                maxes.append(float(r[2]))
            except ValueError:
                continue
            for name, flag in zip(names, r[5:9]):
                if flag.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        loaded = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(maxes), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(layout, steps: int, threads: int, settle_steps: int = 0):
    """The CPU FP64 restatement on `threads` host threads: `settle_steps` untimed, then `steps`
    timed (the same simulated interval the GPU arm times)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    result = oracle.run(layout, settle_steps + steps, (), threads=threads, timed_from=settle_steps)
    if result.status != 0:
        raise RuntimeError(f"oracle failed: {result.message}")
    value = layout.segment_count * steps / (result.run_ms / 1000.0)
    return value, result.run_ms


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
        return float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def recorded_traffic():
    """DRAM bytes per window-kernel launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "window_kernel_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def mixed_accuracy(layout, fp64, mixed, voltage_window_ms, raster_window_ms) -> dict:
    """Mixed mode against FP64 on the same schedule: soma voltages of every cell over
    `voltage_window_ms` and the cell spike raster over `raster_window_ms` (the whole run from
    t = 0, settle included).

    The FP64 path reproduces the CPU FP64 oracle bit for bit (tests/test_parity_gpu.py), so
    these are also the differences to the oracle.  A spike counts as matched when the same cell
    has a spike in the other run within one dt.
    """
    v64, sid64, t64 = fp64
    v32, sid32, t32 = mixed
    dv = np.abs(v32 - v64)
    sub = (v64 < -50.0) & (v32 < -50.0)
    n_cells = layout.n_cells
    dt = layout.dt
    shifts = []
    matched = 0
    cell64 = sid64 < n_cells
    for sid, t in zip(sid64[cell64], t64[cell64]):
        same = t32[sid32 == sid]
        if same.size:
            d = np.min(np.abs(same - t))
            if d <= dt + 1e-9:
                matched += 1
                shifts.append(d)
    n64 = int(np.sum(cell64))
    n32 = int(np.sum(sid32 < n_cells))
    return {
        "reference": "FP64 path (bit-identical to the CPU FP64 oracle)",
        "voltage_window_ms": list(voltage_window_ms), "raster_window_ms": list(raster_window_ms),
        "max_dv_mv": float(dv.max()), "max_dv_subthreshold_mv": float(dv[sub].max()) if sub.any() else None,
        "p99_dv_mv": float(np.percentile(dv, 99)),
        "cell_spikes_fp64": n64, "cell_spikes_mixed": n32,
        "spikes_within_1dt": (matched / n64) if n64 else None,
        "mean_shift_ms": float(np.mean(shifts)) if shifts else None,
    }


def device_timed(fn):
    """fn() bracketed by CUDA events on the current stream (the library's calls are
    synchronous), after a device synchronize and a barrier; returns (result, ms)."""
    import torch
    import torch.distributed as dist

    torch.cuda.synchronize()
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    out = fn()
    stop.record()
    torch.cuda.synchronize()
    return out, start.elapsed_time(stop)


def measure_sharded(args, layout, rank: int, world: int, precision: str, local_rank: int, settle_steps: int = 0):
    """One config-2 network over `world` GPUs: this rank's cells, spikes exchanged per window
    (mind_b200.sharding).  Timed on the device around the window loop, exchanges included;
    the job figure uses the slowest rank.  The settle and warm-up run untimed first."""
    import mind_b200 as mb
    from mind_b200 import replicas, sharding

    # on GPUs the library exchanges the window's spikes itself (NCCL on its stream); the
    # host exchange stands in on the CPU backend
    exchange = "device" if COLLECTIVE_DEVICE == "cuda" else "host"
    run = sharding.ShardedRun(layout, rank, world, precision=precision, device=COLLECTIVE_DEVICE, local=True,
                              exchange=exchange)
    rasters = [run.run_steps(settle_steps, (), True), run.run_steps(args.warmup, (), True)]
    run.launches = 0
    sampler = ClockSampler(local_rank)
    with sampler:
        result, ms = device_timed(lambda: run.run_steps(args.steps, (), True))
    clocks = sampler.summary()
    rasters.append(result)
    launches = run.launches
    run_ms, units = replicas.reduce_timing(ms, layout.segment_count * args.steps, device=COLLECTIVE_DEVICE)
    events = delivered_events(layout, result.spike_sources)
    algo = algorithmic_bytes_per_step(layout, events / args.steps)
    achieved = algo * args.steps / (result.device_ms / 1000.0) / 1e9 if result.device_ms > 0 else None
    soma = run.records([layout.voltage_node(c) for c in range(1, layout.n_cells + 1)])
    rasters.append(run.run_steps(args.steps, soma, True))
    e2e_t0 = run.state.time()[1]
    e2e_result, e2e_ms = device_timed(lambda: run.run_steps(args.steps, soma, True))
    rasters.append(e2e_result)
    e2e_ms, _ = replicas.reduce_timing(e2e_ms, 0.0, device=COLLECTIVE_DEVICE)
    d2h = (len(soma) * 8 * (args.steps + 1) + 16 * len(e2e_result.spike_times)) / args.steps
    run.close()
    trace = np.stack([e2e_result.traces[r.name] for r in soma])
    end_ms = e2e_t0 + args.steps * layout.dt
    return ({"value": units / (run_ms / 1000.0), "ms_per_step": run_ms / args.steps,
             "window_ms": result.device_ms, "window_launches": None, "launches": launches,
             "window_steps": run.window, "bins": None, "algo_bytes_per_step": algo, "achieved_gbs": achieved,
             "spikes": int(len(result.spike_times)), "delivered_events": events,
             "cell_spikes_timed": int(np.sum(result.spike_sources < layout.n_cells)),
             "e2e": units / (e2e_ms / 1000.0), "d2h": d2h, "h2d": 0.0,
             "voltage_window_ms": [e2e_t0, end_ms], "raster_window_ms": [0.0, end_ms],
             "exchange": ("ncclAllGather of (sid, step) blocks per window inside the library, device-resident"
                          if exchange == "device" else "all-gather of (sid, time) per window through the host")},
            (trace, np.concatenate([r.spike_sources for r in rasters]),
             np.concatenate([r.spike_times for r in rasters])), clocks)


def measure_surrogate(args, model, layout, train_ms: float = 300.0, eval_ms: float = 1000.0, keep: float = 0.02,
                      calibration_rounds: int = 4):
    """Config 4 with the surrogate: train on a detailed FP64 run of train_ms, calibrate one
    logit offset per population on the coupled run (calibration_rounds runs of train_ms from
    initialize, towards the training run's population rates over the same window), then run eval_ms from
    initialize twice — plain FP64, and with all but `keep` of the cells replaced — and
    compare time per step and the regions' population rates over the whole eval_ms (which
    extends past the training period)."""
    import mind_b200 as mb
    from mind_b200 import surrogate

    if args.config != 4:
        raise SystemExit("--surrogate needs --config 4")
    macro = model.macro
    t0 = time.perf_counter()
    net, scale, train_run = surrogate.train_from_run(model, train_ms, steps=500, batch=4096)
    train_s = time.perf_counter() - t0
    steps = int(round(eval_ms / layout.dt))
    mb.initialize(model)
    plain, plain_ms = device_timed(lambda: model.state.run_steps(steps, []))
    rng = np.random.default_rng(0)
    mask = rng.uniform(size=layout.n_cells) >= keep
    target_hz = surrogate.population_rates(layout, macro, train_run, train_ms)
    state = mb.runtime.DeviceState(layout, "mixed")   # the tuned mode for the detailed sample
    state.attach_macro(macro)
    state.attach_surrogate(net, mask, scale)
    t_c = time.perf_counter()
    offsets, cal_rates = surrogate.calibrate(state, layout, macro, mask, target_hz, train_ms, calibration_rounds)
    calibration_s = time.perf_counter() - t_c
    state.initialize()
    sur, sur_ms = device_timed(lambda: state.run_steps(steps, []))
    state.close()
    # the same run with the cable solver as judge: populations whose surrogate rate leaves
    # their detailed sample's by more than 5% (plus 3 Poisson standard errors) are reverted
    state = mb.runtime.DeviceState(layout, "mixed")
    state.attach_macro(macro)
    state.attach_surrogate(net, mask, scale)
    state.set_surrogate_offsets(offsets)
    state.initialize()
    t_j = time.perf_counter()
    judged, log, final_mask = surrogate.judged_run(state, layout, macro, mask, eval_ms, window_ms=20.0, bound=0.05)
    judged_wall = (time.perf_counter() - t_j) * 1000.0
    state.close()
    judged_ms = sum(r.device_ms for r in judged)
    # the same with a rotating sample: every cell attached, half of each population's sample
    # exchanged every window (a joining cell counts from its second window)
    state = mb.runtime.DeviceState(layout, "mixed")
    state.attach_macro(macro)
    state.attach_surrogate(net, np.ones(layout.n_cells, dtype=bool), scale)
    state.set_surrogate_cells(mask)
    state.set_surrogate_offsets(offsets)
    state.initialize()
    rotating, rot_log, rot_mask = surrogate.judged_run(state, layout, macro, mask, eval_ms, window_ms=20.0,
                                                       bound=0.05, rotate=True)
    state.close()
    rot_ms = sum(r.device_ms for r in rotating)
    merged = type(plain)(plain.time, {}, np.concatenate([r.spike_times for r in judged]),
                         np.concatenate([r.spike_sources for r in judged]), judged_ms)
    r_judged = surrogate.region_rates(layout, merged, macro, eval_ms)
    merged_rot = type(plain)(plain.time, {}, np.concatenate([r.spike_times for r in rotating]),
                             np.concatenate([r.spike_sources for r in rotating]), rot_ms)
    r_rot = surrogate.region_rates(layout, merged_rot, macro, eval_ms)
    r_plain = surrogate.region_rates(layout, plain, macro, eval_ms)
    r_sur = surrogate.region_rates(layout, sur, macro, eval_ms)
    mean_plain = r_plain.mean(axis=0)
    rel = np.abs(r_sur.mean(axis=0) - mean_plain) / np.maximum(mean_plain, 1e-9)
    rel_j = np.abs(r_judged.mean(axis=0) - mean_plain) / np.maximum(mean_plain, 1e-9)
    rel_r = np.abs(r_rot.mean(axis=0) - mean_plain) / np.maximum(mean_plain, 1e-9)
    # counting noise of two independent runs' rate estimates per region: sqrt(2 / spikes)
    spikes_plain = mean_plain * (eval_ms * 1e-3) * np.bincount(
        surrogate.cell_regions(layout, macro)[surrogate.cell_regions(layout, macro) >= 0], minlength=macro.n_regions)
    noise = np.sqrt(2.0 / np.maximum(spikes_plain, 1.0))
    pooled = abs(r_sur.mean() - r_plain.mean()) / max(r_plain.mean(), 1e-9)
    units = layout.segment_count * steps
    return {
        "metric": "compartment-steps/s (config 4, equivalent: every cell's compartments counted)",
        "config": {"workload": "config4", "cells": layout.n_cells, "compartments": layout.segment_count,
                   "surrogate_cells": int(mask.sum()), "train_ms": train_ms, "eval_ms": eval_ms},
        "plain_fp64": {"value": units / (plain_ms / 1000.0), "ms_per_step": plain_ms / steps},
        "surrogate": {"value": units / (sur_ms / 1000.0), "ms_per_step": sur_ms / steps},
        "speedup": plain_ms / sur_ms,
        "population_rate_error": {"per_region_mean_rel": rel.tolist(), "max_rel": float(rel.max()),
                                  "mean_rel": float(rel.mean()), "pooled_rel": float(pooled),
                                  "counting_noise_per_region_mean": float(noise.mean()),
                                  "plain_rate_hz": mean_plain.tolist(),
                                  "surrogate_rate_hz": r_sur.mean(axis=0).tolist()},
        "judged": {"value": units / (judged_ms / 1000.0), "ms_per_step": judged_ms / steps,
                   "speedup": plain_ms / judged_ms, "wall_ms_with_judge": judged_wall,
                   "reverted": [{"t_ms": t, "regions": regs} for t, regs in log],
                   "surrogate_cells_at_end": int(final_mask.sum()),
                   "population_rate_error": {"mean_rel": float(rel_j.mean()), "max_rel": float(rel_j.max())},
                   "rule": "every 20 ms, over the run so far: |rate(surrogate) - rate(sample)| > 0.05 rate(sample)"
                           " + 3 Poisson standard errors reverts the population"},
        "judged_rotating": {"value": units / (rot_ms / 1000.0), "speedup": plain_ms / rot_ms,
                            "reverted": [{"t_ms": t, "regions": regs} for t, regs in rot_log],
                            "surrogate_cells_at_end": int(rot_mask.sum()),
                            "population_rate_error": {"mean_rel": float(rel_r.mean()), "max_rel": float(rel_r.max())},
                            "rule": "as judged, with half of each population's sample exchanged every window"},
        "calibration": {"rounds": calibration_rounds, "ms_per_round": train_ms, "wall_s": calibration_s,
                        "target_hz": target_hz.tolist(),
                        "surrogate_hz_per_round": [np.nan_to_num(r).tolist() for r in cal_rates],
                        "offsets_per_region": [float(offsets[surrogate.cell_regions(layout, macro) == p][0])
                                               if np.any(surrogate.cell_regions(layout, macro) == p) else 0.0
                                               for p in range(macro.n_regions)]},
        "training": {"windows": int((train_run.drive.shape[0] - surrogate.WINDOW_BINS) * layout.n_cells),
                     "steps": 500, "batch": 4096, "wall_s": train_s},
        "note": "plain: every cell in FP64; surrogate: the detailed sample in the mixed mode, the rest "
                "replaced; regions FP64 in both; rates from the rasters",
    }


def measure_config5(args, model, layout, train_ms: float = 500.0, eval_ms: float = 100.0, keep: float = 0.02,
                    calibration_rounds: int = 4):
    """Config 5 once: a surrogate trained on config 4 (about 1e6 windows of a detailed run of
    train_ms), calibrated on the coupled 100,000-cell run (one offset for all populations,
    rounds of eval_ms from initialize, against the pooled rate of the detailed sample: about
    10 sample cells per population are too few to calibrate each), then eval_ms from
    initialize twice -- every cell detailed
    (mixed mode), and all but `keep` of the cells replaced -- with time per step and the
    regions' population rates."""
    import mind_b200 as mb
    from mind_b200 import networks, surrogate

    macro = model.macro
    m4 = networks.config4()
    mb.build(m4, seed=1)
    t0 = time.perf_counter()
    net, scale, train_run = surrogate.train_from_run(m4, train_ms, steps=500, batch=4096)
    train_s = time.perf_counter() - t0
    windows = int((train_run.drive.shape[0] - surrogate.WINDOW_BINS) * m4.layout.n_cells)
    m4.state.close()
    del train_run, m4
    steps = int(round(eval_ms / layout.dt))
    plain_state = mb.runtime.DeviceState(layout, "mixed")
    plain_state.attach_macro(macro)
    plain_state.initialize()
    plain, plain_ms = device_timed(lambda: plain_state.run_steps(steps, []))
    plain_state.close()
    rng = np.random.default_rng(0)
    mask = rng.uniform(size=layout.n_cells) >= keep
    state = mb.runtime.DeviceState(layout, "mixed")
    state.attach_macro(macro)
    state.attach_surrogate(net, mask, scale)
    t_c = time.perf_counter()
    offsets, _ = surrogate.calibrate(state, layout, macro, mask, None, eval_ms, calibration_rounds, pooled=True)
    calibration_s = time.perf_counter() - t_c
    state.initialize()
    sur, sur_ms = device_timed(lambda: state.run_steps(steps, []))
    state.close()
    net.close()
    r_plain = surrogate.region_rates(layout, plain, macro, eval_ms)
    r_sur = surrogate.region_rates(layout, sur, macro, eval_ms)
    mean_plain = r_plain.mean(axis=0)
    rel = np.abs(r_sur.mean(axis=0) - mean_plain) / np.maximum(mean_plain, 1e-9)
    members = np.bincount(surrogate.cell_regions(layout, macro)[surrogate.cell_regions(layout, macro) >= 0],
                          minlength=macro.n_regions)
    noise = np.sqrt(2.0 / np.maximum(mean_plain * (eval_ms * 1e-3) * members, 1.0))
    units = layout.segment_count * steps
    return {
        "metric": "compartment-steps/s (config 5, equivalent: every cell's compartments counted)",
        "config": {"workload": "config5", "cells": layout.n_cells, "compartments": layout.segment_count,
                   "populations": macro.n_regions, "surrogate_cells": int(mask.sum()), "eval_ms": eval_ms},
        "plain_mixed": {"value": units / (plain_ms / 1000.0), "ms_per_step": plain_ms / steps},
        "surrogate": {"value": units / (sur_ms / 1000.0), "ms_per_step": sur_ms / steps},
        "speedup": plain_ms / sur_ms,
        "population_rate_error": {"mean_rel": float(rel.mean()), "max_rel": float(rel.max()),
                                  "pooled_rel": float(abs(r_sur.mean() - r_plain.mean()) / max(r_plain.mean(), 1e-9)),
                                  "counting_noise_per_region_mean": float(noise.mean()),
                                  "plain_rate_hz_mean": float(mean_plain.mean()),
                                  "surrogate_rate_hz_mean": float(r_sur.mean())},
        "calibration": {"rounds": calibration_rounds, "ms_per_round": eval_ms, "wall_s": calibration_s,
                        "offset": float(offsets[0]) if len(offsets) else 0.0,
                        "target": "the pooled rate of the detailed sample (all populations), over the rounds"},
        "training": {"source": "config 4 (2,000 cells), detailed FP64 run", "train_ms": train_ms,
                     "windows": windows, "steps": 500, "batch": 4096, "wall_s": train_s},
        "note": "plain: every cell in the mixed mode; surrogate: the detailed sample in the mixed mode, the rest "
                "replaced; regions FP64 in both; rates from the rasters",
    }


def run_reference(args, rank: int):
    """The reference arm: the CPU FP64 restatement of MIND.jl's step loop (oracle/) on every host
    core, on the GPU arm's network and schedule -- the same untimed settle and warm-up, then
    the same --steps timed."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    model, layout = build_network(args.cells, seed=1, config=args.config)
    settle_steps = int(round(args.settle_ms / layout.dt))
    steps = max(1, args.steps)
    value, ms = cpu_baseline(layout, steps, threads, settle_steps + args.warmup)
    line = {
        "impl": "reference", "metric": WORKLOAD_METRICS.get(args.config, METRIC), "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": f"synthetic (seeded config-{args.config} network, mind_b200.networks.config{args.config})",
        "config": {"workload": f"config{args.config}", "cells": layout.n_cells, "compartments": layout.segment_count,
                   "nodes": layout.n_nodes, "dt_ms": layout.dt, "t_start_ms": args.settle_ms,
                   "l2": "state larger than L2"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{steps} micro steps of the full config-{args.config} network from "
                                   f"t = {args.settle_ms:g} ms + {args.warmup} warm-up steps (settle untimed)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "MIND.jl is Julia (absent here) and has no CPU path; the reference arm is the CPU FP64 "
                "restatement of its step loop, every cell's currents, cable solve and state advance "
                "spread over a pool of host threads",
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch

    torch.cuda.set_device(local_rank % torch.cuda.device_count())
    dist = None
    global COLLECTIVE_DEVICE
    if world > 1:
        import datetime

        import torch.distributed as dist

        # NCCL between GPUs; MIND_BENCH_BACKEND=gloo exercises the same exchange with host
        # tensors (e.g. several ranks sharing one GPU in a test).
        backend = os.environ.get("MIND_BENCH_BACKEND", "nccl")
        COLLECTIVE_DEVICE = "cuda" if backend == "nccl" else "cpu"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))

    import mind_b200 as mb
    from mind_b200 import replicas

    model, layout = build_network(args.cells, seed=replicas.replica_seed(1, rank), config=args.config,
                                  rank=rank, world=world)
    sharded = world > 1 and args.config == 2
    if args.config == 5 and not args.surrogate:
        raise SystemExit("--config 5 runs with --surrogate")
    if args.surrogate:
        if rank == 0:
            measure = measure_config5 if args.config == 5 else measure_surrogate
            extra = {} if args.eval_ms is None else {"eval_ms": float(args.eval_ms)}
            print(json.dumps(measure(args, model, layout, **extra)), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    if args.accuracy_ms > 0:
        if rank == 0:
            soma_all = [mb.RecordSpec(layout.voltage_node(c), f"v{c}") for c in range(1, layout.n_cells + 1)]
            runs = {}
            for precision in ("fp64", "mixed"):
                mb.initialize(model, precision=precision)
                r = mb.run(model, args.accuracy_ms, records=soma_all, record_spikes=True)
                runs[precision] = (np.stack([r.traces[x.name] for x in soma_all]), r.spike_sources, r.spike_times)
            steps = int(round(args.accuracy_ms / layout.dt))
            print(json.dumps({"config": f"config{args.config}", "cells": layout.n_cells,
                              "accuracy": mixed_accuracy(layout, runs["fp64"], runs["mixed"], [0.0, args.accuracy_ms],
                                                         [0.0, args.accuracy_ms])}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    soma = [mb.RecordSpec(layout.voltage_node(c), f"v{c}") for c in range(1, layout.n_cells + 1)]
    precisions = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    dt = layout.dt
    settle_steps = int(round(args.settle_ms / dt))
    results, runs = {}, {}
    clocks = None
    for precision in precisions:
        if sharded:
            results[precision], runs[precision], clocks = measure_sharded(args, layout, rank, world, precision,
                                                                          local_rank, settle_steps)
            continue
        mb.initialize(model, precision=precision)
        # launch shape per size bin, timed on trial windows before the measurement (setup,
        # like the build; the state restarts at t = 0)
        shapes = mb.autotune(model, windows=3) if not args.no_autotune else model.state.bin_threads()
        # settle, then warm up, untimed: the timed steps start at t_start on an active network
        rasters = [mb.run(model, settle_steps * dt, record_spikes=True)]
        rasters.append(mb.run(model, (settle_steps + args.warmup) * dt, record_spikes=True))
        model.state.set_profiling(True)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        sampler = ClockSampler(local_rank)
        with sampler:
            result = mb.run(model, (settle_steps + args.warmup + args.steps) * dt, record_spikes=True)
            torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        rasters.append(result)
        model.state.set_profiling(False)
        stats = model.state.run_stats()
        clocks = sampler.summary()
        run_ms, units = replicas.reduce_timing(stats.run_ms, layout.segment_count * args.steps, device=COLLECTIVE_DEVICE)
        value = units / (run_ms / 1000.0)
        events = delivered_events(layout, result.spike_sources)
        algo = algorithmic_bytes_per_step(layout, events / args.steps)
        window_ms = stats.window_ms
        achieved = algo * args.steps / (window_ms / 1000.0) / 1e9 if window_ms > 0 else None
        # End to end through the public API, continuing the same run: one untimed call with the
        # soma records (the library uploads their tables once and keeps them), then the timed
        # call, which copies every soma trace and the raster to the host.
        t_now = model.state.time()[1]
        rasters.append(mb.run(model, t_now + args.steps * dt, records=soma, record_spikes=True))
        e2e_t0 = model.state.time()[1]
        e2e_result, e2e_ms = device_timed(
            lambda: mb.run(model, e2e_t0 + args.steps * dt, records=soma, record_spikes=True))
        rasters.append(e2e_result)
        e2e_ms, _ = replicas.reduce_timing(e2e_ms, 0.0, device=COLLECTIVE_DEVICE)
        e2e_s = e2e_ms / 1000.0
        d2h = (len(soma) * 8 * (args.steps + 1) + 16 * len(e2e_result.spike_times)) / args.steps
        h2d = 0.0   # the record set is unchanged since the untimed call: nothing is uploaded
        runs[precision] = (e2e_result.traces.by_record,
                           np.concatenate([r.spike_sources for r in rasters]),
                           np.concatenate([r.spike_times for r in rasters]))
        results[precision] = {
            "bin_threads": shapes,
            "value": value, "ms_per_step": run_ms / args.steps, "window_ms": window_ms,
            "window_launches": stats.window_launches, "launches": stats.launches, "window_steps": stats.window_steps,
            "bins": stats.bins, "algo_bytes_per_step": algo, "achieved_gbs": achieved,
            "spikes": int(len(result.spike_times)), "delivered_events": events,
            "cell_spikes_timed": int(np.sum(result.spike_sources < layout.n_cells)),
            "e2e": units / e2e_s, "e2e_ms_per_step": e2e_ms / args.steps, "d2h": d2h, "h2d": h2d,
            "voltage_window_ms": [e2e_t0, e2e_t0 + args.steps * dt],
            "raster_window_ms": [0.0, e2e_t0 + args.steps * dt],
        }
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    head = results[precisions[0]]
    peak, peak_kind = measured_peaks()
    traffic = recorded_traffic()
    line = {
        "metric": WORKLOAD_METRICS.get(args.config, METRIC), "value": head["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if precisions[0] == "fp64" else "f32-gating/f64-cable",
        "data": f"synthetic (seeded config-{args.config} network, mind_b200.networks.config{args.config})",
        "config": {"workload": f"config{args.config}", "cells": layout.n_cells, "compartments": layout.segment_count,
                   "nodes": layout.n_nodes, "dt_ms": layout.dt, "precision": precisions[0],
                   "parallelism": (f"cells sharded over {world} GPUs, spike all-gather per window" if sharded
                                   else f"replica x{world}" if world > 1 else "1 GPU"),
                   "l2": "working set larger than L2 (no flush needed)",
                   "window_steps": head["window_steps"], "size_bins": head["bins"],
                   "threads_per_cell_by_bin": head.get("bin_threads"), "t_start_ms": args.settle_ms,
                   "timed_cell_spikes": head.get("cell_spikes_timed")},
        "e2e": {"value": head["e2e"], "unit": UNIT, "h2d_bytes_per_step": head["h2d"],
                "d2h_bytes_per_step": head["d2h"]},
        "roofline": {
            "bound": "hbm",
            "achieved": head["achieved_gbs"], "peak": peak, "unit": "GB/s",
            "frac": (head["achieved_gbs"] / peak) if head["achieved_gbs"] else None,
            "traffic": traffic.get("dram_bytes_per_step") if traffic and args.config == 2 else None,
            "traffic_unit": "DRAM bytes per micro step (all bins of a window / window steps), from one ncu capture",
            "kernel": "window_kernel", "algo_bytes_per_step": head["algo_bytes_per_step"],
            "peak_source": f"{peak_kind} hbm_gbs",
            "note": "achieved = algorithmic bytes of one pass per step / device time per step; the window "
                    "kernel keeps each cell on-chip for a window of steps, so its DRAM traffic (traffic) is "
                    "far below the algorithmic bytes and the kernel is latency-bound, not HBM-bound",
        },
        "gpu_launches": head["launches"],
        "clocks": clocks,
        "modes": {k: {"value": v["value"], "ms_per_step": v["ms_per_step"], "e2e": v["e2e"],
                      "threads_per_cell_by_bin": v.get("bin_threads")}
                  for k, v in results.items()},
        "accuracy": (mixed_accuracy(layout, runs["fp64"], runs["mixed"], head["voltage_window_ms"],
                                    head["raster_window_ms"])
                     if "fp64" in runs and "mixed" in runs else None),
        "spikes": head["spikes"],
    }
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cpu_value, _ = cpu_baseline(layout, args.cpu_steps, threads, settle_steps)
        line["cpu_baseline"] = {"value": cpu_value, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{args.cpu_steps} micro steps of the full config-{args.config} network "
                                          f"from t = {args.settle_ms:g} ms (after an untimed settle)"}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
