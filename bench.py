#!/usr/bin/env python
"""Benchmark of the solver-2d explicit step on B200.

Workload: the 4096 x 4096 synthetic valley flood (dx = 5 m; seeded DEM with a
0.005 longitudinal slope, 0.05 side slopes and 200 Gaussian hills; Manning n
from 4 Voronoi land-cover patches; rain 50 mm/h; point inflow with a
triangular 500 m^3/s hydrograph; transmissive sides; CFL 0.5; SSP-RK2 +
Manning friction + forcings every step). A step advances every cell once:
metric = cell-updates/s. Inputs (~0.67 GB resident) exceed the 126 MB L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun as independent replicas (the grid fits one GPU;
there is no data-path collective); the barrier and the max-over-ranks timing
use torch.distributed. Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
UNIT = "cell-updates/s"
GRID = 4096
DX = 5.0
ALG_BYTES_PER_CELL_UPDATE = 144.0  # stage 1: 32 in + 24 out; stage 2: 64 in + 24 out
STAGE_LAUNCHES_PER_STEP = 2


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=GRID, help="grid side (default 4096)")
    p.add_argument("--cpu-steps", type=int, default=2, help="oracle steps in the CPU baseline")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--stage-kernel", default="auto", choices=["auto", "tile", "tile32", "strip"],
                   help="valley: the stage kernel (hf_sim_set_stage_kernel; bit-identical)")
    p.add_argument("--workload", default="valley", choices=["valley", "ensemble", "adjoint",
                                                            "serve", "lanes", "regimes"],
                   help="valley: the 4096^2 plain step (default line); ensemble: batched "
                        "uneven-size scenarios vs a loop of per-scenario solves; adjoint: "
                        "misfit gradient w.r.t. the Manning field vs the forward solve; "
                        "serve: an arrival stream through the continuous-batching server vs "
                        "a sequential plain solve per request; lanes: zonal Manning "
                        "derivatives in vector mode vs scalar Dual runs vs the adjoint; "
                        "regimes: the reference's criterion step regimes (all wet, mostly "
                        "dry) scaled to --n")
    p.add_argument("--calib-n", type=int, default=512, help="adjoint: grid side")
    p.add_argument("--calib-steps", type=int, default=2000, help="adjoint: steps of the misfit")
    p.add_argument("--checkpoint-every", type=int, default=45)
    p.add_argument("--requests", type=int, default=200, help="serve: requests in the stream")
    p.add_argument("--rate", type=float, default=50.0, help="serve: arrivals per second")
    p.add_argument("--sides", default="64,128,256,512", help="serve: grid sides (uniform)")
    p.add_argument("--horizon", default="60,300", help="serve: horizon range in s (uniform)")
    p.add_argument("--max-active-cells", type=int, default=1 << 20,
                   help="serve: cells advancing together (admission cap)")
    p.add_argument("--no-fifo", action="store_true",
                   help="serve: skip the uncapped FIFO run of the server")
    p.add_argument("--scenarios", type=int, default=512)
    p.add_argument("--loop-every", type=int, default=8,
                   help="ensemble: the per-scenario loop times every k-th scenario")
    p.add_argument("--complete", action="store_true",
                   help="ensemble: also run the batch to every scenario's horizon")
    return p.parse_args()


# --------------------------------------------------------------------- dist
from hydroflux_b200.dist import Dist  # noqa: E402  (ranks, barrier, max over ranks, sharding)


# ------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# The stage kernel in use, as named in the committed ncu summaries.
KERNEL_NAMES = {"tile": "k_stage_pf/32x8", "tile32": "k_stage_pf/32x32", "strip": "k_stage_strip"}


def profiled_figure(kernel, key):
    """A per-cell figure of a stage kernel from the committed ncu summary
    (lines `<kernel>.<key>: value`)."""
    path = os.path.join(ROOT, "profiles", "stage_kernel_traffic.txt")
    try:
        for line in open(path):
            if line.startswith(f"{kernel}.{key}:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def profiled_traffic(kernel):
    """DRAM bytes per stage launch per cell from the committed ncu summary."""
    return profiled_figure(kernel, "dram_bytes_per_cell_per_launch")


def issue_roof(kernel, value, clk):
    """The bound the stage kernel actually runs against: instruction issue.
    Warp instructions per cell-update from the committed ncu summary; the
    peak issues one warp instruction per scheduler per cycle (4 per SM) on
    every SM at the SM clock measured during the timed region."""
    per_cell = profiled_figure(kernel, "warp_instructions_per_cell_update")
    if per_cell is None or not clk or not clk.get("sm_mhz"):
        return None
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    peak = sms * 4 * clk["sm_mhz"] * 1e6 / per_cell
    return {"unit": UNIT, "achieved": value, "peak": peak, "frac": value / peak,
            "warp_instructions_per_cell_update": per_cell, "sms": sms, "sm_mhz": clk["sm_mhz"]}


# ---------------------------------------------------------------- workload
def valley_config(a, world, wet_frac):
    """The `config` of the plain-step line; both arms print the same dict."""
    return {"workload": f"valley flood {a.n}x{a.n}, dx=5 m, SSP-RK2 + Manning + rain + "
                        f"point inflow, CFL 0.5, transmissive sides",
            "grid": f"{a.n}x{a.n}", "cells": a.n * a.n, "integrator": "ssprk2",
            "wet_fraction": round(wet_frac, 4),
            "l2": "inputs larger than L2 (h,hu,hv,z,n = 40 B/cell resident)",
            "parallelism": f"replicas x{world}" if world > 1 else "single grid"}


def make_workload(n):
    from hydroflux_b200 import workloads
    return workloads.valley(n=n, dx=DX, seed=0)


def cpu_baseline(scn, state, t0, steps, threads):
    """Oracle (CPU restatement of the reference) on `steps` steps of the same
    workload from the same state; returns cell-updates/s."""
    from hydroflux_b200 import abi, workloads
    from oracle import oracle as O
    O.set_threads(threads)
    cfg = abi.make_config(cfl=scn.cfl, boundaries=abi.make_boundaries(*scn.bcs), max_dt=scn.max_dt)
    f = workloads.oracle_forcing(scn)
    h, hu, hv = state
    t_start = time.perf_counter()
    r = O.sim_run(scn.bed, scn.manning, scn.dx, scn.dy, h, hu, hv, cfg, scn.t_end, forcing=f,
                  stop_after=steps, t0=t0)
    el = time.perf_counter() - t_start
    assert r["status"] == 0, r["message"]
    done = r["steps"]
    return scn.n_cells * done / el, el, done


# -------------------------------------------------------------- ours (GPU)
def launches() -> int:
    """Kernels the library has launched so far in this process (its own
    count: direct launches plus every kernel node of each graph launch)."""
    from hydroflux_b200 import _lib
    return _lib.kernel_launches()


def run_ours(a, d: Dist):
    import torch

    from hydroflux_b200 import _lib, workloads
    dev = d.local
    torch.cuda.set_device(dev)
    _lib.lib()
    scn = make_workload(a.n)
    cells = scn.n_cells

    sm = workloads.simulation_for(scn, device=dev)
    sm.set_stage_kernel(a.stage_kernel)
    h_d, hu_d, hv_d, stream_ptr = sm.device_state()
    stream = torch.cuda.ExternalStream(stream_ptr, device=dev)
    sm.run_steps(max(a.warmup, 3), scn.t_end)
    torch.cuda.synchronize(dev)
    warm_t = sm.time()
    # Snapshot of the warmed state (pinned host) for the e2e and CPU legs.
    pinned = [torch.empty(scn.shape, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    for p_, t_ in zip(pinned, (h_d, hu_d, hv_d)):
        p_.copy_(t_)
    wet_frac = float((pinned[0] > 1e-6).double().mean())

    # ---- timed region: K steps replayed from CUDA-graph chunks
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.3)
    d.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
    k_launch = launches()
    sm.run_steps(a.steps, scn.t_end)
    k_launch = launches() - k_launch
    with torch.cuda.stream(stream):
        e1.record(stream)
    torch.cuda.synchronize(dev)
    d.barrier()
    clk = clocks.stop()
    ms_local = e0.elapsed_time(e1)
    ms = d.max(ms_local)
    steps_done = a.steps
    value = d.world * cells * steps_done / (ms / 1e3)

    # ---- stage-kernel timing for the roofline (events around every stage launch)
    stage_ms, stage_launches, region_ms = sm.run_steps_timed(a.steps, scn.t_end)
    stage_ms = d.max(stage_ms)
    avg_stage_s = stage_ms / 1e3 / max(stage_launches, 1)
    bytes_per_launch = ALG_BYTES_PER_CELL_UPDATE / STAGE_LAUNCHES_PER_STEP * cells
    achieved_gbs = bytes_per_launch / avg_stage_s / 1e9
    peak, peak_kind = measured_peaks()
    kernel = KERNEL_NAMES[sm.stage_kernel()]
    traffic_per_cell = profiled_traffic(kernel)
    sm.close()

    # ---- e2e: through the C ABI with host buffers (pinned), copies timed
    e2e = None
    if not a.no_e2e:
        from hydroflux_b200 import sim as S
        scn_w = scn
        bed_p = torch.from_numpy(scn.bed).pin_memory()
        man_p = torch.from_numpy(scn.manning).pin_memory()
        # the caller's pinned result buffers, allocated once like the inputs
        out = [torch.empty(scn.shape, dtype=torch.float64, pin_memory=True) for _ in range(3)]
        torch.cuda.synchronize(dev)
        d.barrier()
        t_a = time.perf_counter()
        cfg = S.SimulationConfig(cfl=scn_w.cfl, boundaries=S.Boundaries2D(
            *[S.Boundary(k, v) for k, v in scn_w.bcs]), max_dt=scn_w.max_dt)
        mesh = S.Mesh2D(bed_p.numpy(), scn_w.dx, scn_w.dy, man_p.numpy())
        st = tuple(p_.numpy() for p_ in pinned)
        s2 = S.Simulation(mesh, st, cfg, dev)
        s2.set_stage_kernel(a.stage_kernel)
        s2.set_rain(np.stack(scn_w.rain, axis=1))
        s2.set_point_sources([S.PointSource(r, c, np.stack([t, q], axis=1))
                              for r, c, t, q in scn_w.sources])
        t_c = time.perf_counter()
        for _ in range(a.steps):
            s2.step(scn_w.t_end - s2.time())
        t_s = time.perf_counter()
        from hydroflux_b200._lib import lib as _l
        rc = _l().hf_sim_get_state(s2._h, out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr())
        assert rc == 0
        t_b = time.perf_counter()
        s2.close()
        el = d.max(t_b - t_a)
        h2d = (5 * cells * 8 + 64) / a.steps
        d2h = (3 * cells * 8) / a.steps + 128
        e2e = {"value": d.world * cells * a.steps / el, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "create_ms": 1e3 * (t_c - t_a), "steps_ms": 1e3 * (t_s - t_c),
               "readback_ms": 1e3 * (t_b - t_s),
               "note": "Simulation::new from pinned host arrays (bed, n, h, hu, hv), K x "
                       "Simulation::step through the C ABI (dt read back each step), "
                       "states() to pinned host; copies, allocation (from the library's "
                       "device pool, which keeps the memory of the destroyed timed-leg "
                       "handle) and graph capture timed"}

    cpu = None
    if d.rank == 0 and d.world == 1 and not a.no_cpu_baseline:
        st = tuple(p_.numpy().copy() for p_ in pinned)
        v, el, done = cpu_baseline(scn, st, warm_t, a.cpu_steps, 1)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{done} steps of the same 4096^2 workload from the warmed state "
                         f"(wet fraction {wet_frac:.3f}), CPU oracle (C++ restatement of the "
                         f"reference's serial path), 1 thread, {el:.1f} s"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": d.world, "steps": a.steps,
        "warmup": max(a.warmup, 3), "ms_per_step": ms / steps_done, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded valley DEM, Voronoi Manning field, rain + inflow hydrograph)",
        "config": valley_config(a, d.world, wet_frac),
        "e2e": e2e,
        "gpu_launches": k_launch,
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                     "frac": achieved_gbs / peak, "peak_source": peak_kind,
                     "traffic": (traffic_per_cell * cells) if traffic_per_cell else None,
                     "kernel": kernel, "alg_bytes_per_launch": bytes_per_launch,
                     "avg_launch_ms": avg_stage_s * 1e3, "launches": stage_launches,
                     "issue": issue_roof(kernel, value / d.world, clk)},
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    if d.rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------ reference arm (CPU)
def run_reference(a, d: Dist):
    """The reference's CPU path (the oracle: C++ restatement of its serial
    step, OpenMP row chunks like its rayon feature) on the same workload, the
    same warm-up (max(W, 3) steps from the dry start) and the same K timed
    steps as the GPU arm; only rank 0 runs it."""
    if d.rank != 0:
        return
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    scn = make_workload(a.n)
    cells = scn.n_cells
    from hydroflux_b200 import abi, workloads
    cfg = abi.make_config(cfl=scn.cfl, boundaries=abi.make_boundaries(*scn.bcs), max_dt=scn.max_dt)
    f = workloads.oracle_forcing(scn)
    O.set_threads(threads)
    warm = max(a.warmup, 3)
    r = O.sim_run(scn.bed, scn.manning, scn.dx, scn.dy, scn.h, scn.hu, scn.hv, cfg, scn.t_end,
                  forcing=f, stop_after=warm)
    assert r["status"] == 0, r["message"]
    wet_frac = float(np.mean(r["h"] > 1e-6))
    t0 = time.perf_counter()
    r2 = O.sim_run(scn.bed, scn.manning, scn.dx, scn.dy, r["h"], r["hu"], r["hv"], cfg,
                   scn.t_end, forcing=f, stop_after=a.steps, t0=r["t"], steps0=r["steps"])
    el = time.perf_counter() - t0
    assert r2["status"] == 0, r2["message"]
    k = r2["steps"] - r["steps"]
    value = cells * k / el
    sample = (f"all {k} timed steps on the full {a.n}^2 workload after {warm} warm-up steps "
              f"from the dry start; CPU oracle (C++ restatement of the reference, OpenMP row "
              f"chunks like its rayon feature), {threads} threads, {el:.1f} s")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": k,
            "warmup": warm, "ms_per_step": el / k * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded valley DEM, Voronoi Manning field, rain + inflow hydrograph)",
            "config": valley_config(a, d.world, wet_frac),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_regimes(a, d: Dist):
    """The reference's criterion regimes of the step (solver-2d/benches/
    step.rs:44-75) at --n (default 4096^2): the mostly-dry valley (6.25%
    wet, where the dry-cell paths dominate) and the all-wet flat bed, each
    K steps of Simulation::step (SSP-RK2 + Manning, walls) timed with CUDA
    events; the oracle (1 thread) times one step of each beside it.
    Replicas on N > 1."""
    import torch

    from hydroflux_b200 import _lib, abi, workloads
    from oracle import oracle as O
    dev = d.local
    torch.cuda.set_device(dev)
    _lib.lib()
    out = {}
    clocks = ClockSampler(dev)
    clocks.start()
    k_launch = 0
    for kind in ("mostly_dry", "all_wet"):
        scn = workloads.step_regime(kind, a.n)
        with workloads.simulation_for(scn, device=dev) as sm:
            h_d, _, _, stream_ptr = sm.device_state()
            stream = torch.cuda.ExternalStream(stream_ptr, device=dev)
            sm.run_steps(max(a.warmup, 3))
            torch.cuda.synchronize(dev)
            wet = float((h_d > 1e-6).double().mean())
            d.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
            k0 = launches()
            sm.run_steps(a.steps)
            k_launch += launches() - k0
            with torch.cuda.stream(stream):
                e1.record(stream)
            torch.cuda.synchronize(dev)
            ms = d.max(e0.elapsed_time(e1))
            kernel = sm.stage_kernel()
            state = sm.states()
            t0 = sm.time()
        cpu = None
        if d.rank == 0 and d.world == 1 and not a.no_cpu_baseline:
            O.set_threads(1)
            cfg = abi.make_config(cfl=scn.cfl, boundaries=abi.make_boundaries(*scn.bcs),
                                  max_dt=scn.max_dt)
            tc = time.perf_counter()
            r = O.sim_run(scn.bed, scn.manning, scn.dx, scn.dy, *state, cfg, scn.t_end,
                          stop_after=1, t0=t0)
            el = time.perf_counter() - tc
            assert r["status"] == 0, r["message"]
            cpu = {"value": scn.n_cells / el, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": "1 step of the same state, CPU oracle, 1 thread"}
        out[kind] = {"value": d.world * scn.n_cells * a.steps / (ms / 1e3), "unit": UNIT,
                     "ms_per_step": ms / a.steps, "wet_fraction": round(wet, 4),
                     "stage_kernel": KERNEL_NAMES[kernel],
                     "cpu_baseline": cpu}
    clk = clocks.stop()
    line = {"metric": "cell-updates/s (mostly dry)", "value": out["mostly_dry"]["value"],
            "unit": UNIT, "n_gpus": d.world, "steps": a.steps, "warmup": max(a.warmup, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the reference's criterion regimes, scaled)",
            "config": {"workload": f"solver-2d/benches/step.rs regimes at {a.n}x{a.n}, dx 1 m, "
                                   "SSP-RK2 + Manning 0.03, walls, CFL 0.4",
                       "l2": "inputs larger than L2" if a.n >= 2048 else "L2-resident",
                       "parallelism": f"replicas x{d.world}" if d.world > 1 else "single grid"},
            "regimes": out,
            "mostly_dry_vs_all_wet": out["mostly_dry"]["value"] / out["all_wet"]["value"],
            "gpu_launches": k_launch, "clocks": clk}
    if d.rank == 0:
        print(json.dumps(line), flush=True)


def run_ensemble(a, d: Dist):
    """Batched ensemble (hf_batch_*) against a loop of per-scenario plain GPU
    solves (hf_sim run_steps, one scenario after another), same scenarios and
    the same number of steps per scenario. Scenarios are sharded over ranks by
    cell count (longest first to the lightest rank; no collective)."""
    import torch

    from hydroflux_b200 import _lib, workloads
    from hydroflux_b200.ensemble import Ensemble, ensemble_scenarios
    dev = d.local
    torch.cuda.set_device(dev)
    _lib.lib()
    t_gen = time.perf_counter()
    allscn = ensemble_scenarios(count=a.scenarios, seed=0)
    mine = [allscn[i] for i in d.shard([s.n_cells for s in allscn])]
    gen_s = time.perf_counter() - t_gen
    if a.complete:
        return run_ensemble_complete(a, d, allscn, mine, gen_s)
    cells = np.array([s.n_cells for s in mine], dtype=np.float64)
    ens = Ensemble(mine, device=dev)
    ens.run(max(a.warmup, 3))
    ens.run(64)  # untimed: the tile-schedule autotuner times 2 x 4 chunks of 8 steps
    sched, tune_ms = ens.schedule()
    st0 = np.array([ens.info(k)["steps"] for k in range(len(mine))], dtype=np.float64)
    torch.cuda.synchronize(dev)
    d.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    k_launch = launches()
    t0 = time.perf_counter()
    left = ens.run(a.steps)
    t1 = time.perf_counter()
    k_launch = launches() - k_launch
    clk = clocks.stop()
    st1 = np.array([ens.info(k)["steps"] for k in range(len(mine))], dtype=np.float64)
    el = d.max(t1 - t0)
    batched = float(np.sum(cells * (st1 - st0)))
    batched_rate = d.sum(batched) / el
    ens.close()
    # Loop of per-scenario plain solves on a subset, same steps per scenario.
    sub = mine[::max(a.loop_every, 1)]
    loop_cells, loop_time = 0.0, 0.0
    for s in sub:
        sm = workloads.simulation_for(s, device=dev)
        sm.run_steps(max(a.warmup, 3), s.t_end)
        torch.cuda.synchronize(dev)
        k0 = sm.steps()
        ta = time.perf_counter()
        sm.run_steps(a.steps, s.t_end)
        tb = time.perf_counter()
        loop_cells += s.n_cells * (sm.steps() - k0)
        loop_time += tb - ta
        sm.close()
    loop_rate = loop_cells / loop_time if loop_time > 0 else None
    line = {"metric": "ensemble cell-updates/s (batched)", "value": batched_rate,
            "unit": "cell-updates/s", "n_gpus": d.world, "steps": a.steps,
            "warmup": max(a.warmup, 3), "higher_is_better": True, "scaling": "strong",
            "dtype": "f64", "data": "synthetic (seeded valley ensemble)",
            "config": {"workload": f"{a.scenarios} scenarios, side log-uniform in [64, 1024], "
                                   "valley DEM per-scenario seed, n ~ U[0.02, 0.08], inflow "
                                   "peak 500 x U[0.5, 2] m^3/s, horizon 30 min, dx 5 m",
                       "cells": int(sum(s.n_cells for s in allscn)),
                       "parallelism": f"scenarios sharded over {d.world} GPU(s)"},
            "loop_of_plain_solves": {"value": loop_rate, "unit": "cell-updates/s",
                                     "scenarios_timed": len(sub)},
            "speedup_vs_loop": (batched_rate / d.world) / loop_rate if loop_rate else None,
            "gpu_launches": k_launch, "generation_s": gen_s,
            "schedule": {"chosen": Ensemble.SCHEDULES.get(sched, "untuned"),
                         "tuning_ms_per_candidate": [float(x) for x in tune_ms],
                         "autotune_steps": 64},
            "clocks": clk}
    if d.rank == 0:
        print(json.dumps(line), flush=True)


def run_ensemble_complete(a, d: Dist, allscn, mine, gen_s):
    """Config 3 as its metric states: every scenario solved to its 30-min
    horizon, batched (one hf_batch handle, run until all have finished)
    against a loop of plain per-scenario solves (hf_sim run_until, one after
    another), solves/s of each. The first --scenarios scenarios of the
    seeded sequence (the same log-uniform side distribution); handle
    creation and uploads are outside both timings."""
    import torch

    from hydroflux_b200 import workloads
    from hydroflux_b200.ensemble import Ensemble
    dev = d.local
    # untimed warm-up: one small scenario through each path (module load,
    # kernel attributes, graph capture)
    warm = [dataclasses.replace(allscn[0], t_end=30.0)]
    with Ensemble(warm, device=dev) as e:
        e.run()
    with workloads.simulation_for(warm[0], device=dev) as sm:
        sm.run_until(warm[0].t_end)
    torch.cuda.synchronize(dev)
    d.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    ens = Ensemble(mine, device=dev)
    torch.cuda.synchronize(dev)
    k_batch = launches()
    t0 = time.perf_counter()
    left = ens.run()
    torch.cuda.synchronize(dev)
    batch_s = time.perf_counter() - t0
    k_batch = launches() - k_batch
    info = [ens.info(k) for k in range(len(mine))]
    sched, _ = ens.schedule()
    ens.close()
    loop_s, loop_steps = [], []
    k_loop = 0
    for s in mine:
        with workloads.simulation_for(s, device=dev) as sm:
            torch.cuda.synchronize(dev)
            k0 = launches()
            ta = time.perf_counter()
            sm.run_until(s.t_end)
            torch.cuda.synchronize(dev)
            loop_s.append(time.perf_counter() - ta)
            k_loop += launches() - k0
            loop_steps.append(sm.steps())
    clk = clocks.stop()
    steps = np.array([x["steps"] for x in info], dtype=np.float64)
    ok = sum(1 for x in info if x["status"] == 0)
    cells = np.array([s.n_cells for s in mine], dtype=np.float64)
    tot = d.gather({"n": len(mine), "ok": ok, "batch_s": batch_s, "loop_s": float(sum(loop_s)),
                    "cell_updates": float(np.sum(cells * steps)),
                    "same_steps": bool(np.array_equal(steps, np.array(loop_steps))),
                    "steps": steps.tolist(), "sides": [s.shape[0] for s in mine],
                    "loop_each": loop_s, "k_batch": k_batch, "k_loop": k_loop})
    if d.rank != 0:
        return
    n_all = sum(x["n"] for x in tot)
    b_s = max(x["batch_s"] for x in tot)
    l_s = max(x["loop_s"] for x in tot)
    st = np.concatenate([np.array(x["steps"]) for x in tot])
    sides = np.concatenate([np.array(x["sides"]) for x in tot])
    each = np.concatenate([np.array(x["loop_each"]) for x in tot])
    small = sides <= 256
    line = {"metric": "ensemble solves/s to the horizon (batched)", "value": n_all / b_s,
            "unit": "solves/s", "n_gpus": d.world, "steps": int(st.max()), "warmup": 1,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded valley ensemble)",
            "config": {"workload": f"the first {a.scenarios} of the seeded 512-scenario ensemble: "
                                   "side log-uniform in [64, 1024], valley DEM per-scenario "
                                   "seed, n ~ U[0.02, 0.08], inflow peak 500 x U[0.5, 2] m^3/s, "
                                   "horizon 30 min each, dx 5 m",
                       "scenarios": n_all, "cells": int(sum(s.n_cells for s in allscn)),
                       "parallelism": f"scenarios sharded over {d.world} GPU(s)"},
            "batched_s": b_s, "scenarios_completed": sum(x["ok"] for x in tot),
            "unfinished": left,
            "loop_of_plain_solves": {"value": n_all / l_s, "unit": "solves/s", "seconds": l_s,
                                     "steps_equal_batched": all(x["same_steps"] for x in tot),
                                     "gpu_launches": sum(x["k_loop"] for x in tot)},
            "speedup_vs_loop": l_s / b_s,
            "cell_updates": sum(x["cell_updates"] for x in tot),
            "batched_cell_updates_per_s": sum(x["cell_updates"] for x in tot) / b_s,
            "steps_per_scenario": {"min": int(st.min()), "median": float(np.median(st)),
                                   "max": int(st.max())},
            "loop_time_share_sides_le_256": float(each[small].sum() / max(each.sum(), 1e-30)),
            "schedule": Ensemble.SCHEDULES.get(sched, "untuned"),
            "generation_s": gen_s, "gpu_launches": sum(x["k_batch"] for x in tot),
            "clocks": clk}
    print(json.dumps(line), flush=True)


def run_adjoint(a, d: Dist):
    """Gradient of the gauge misfit with respect to the per-cell Manning field
    (hf_grad_manning, checkpointed adjoint) against the forward solve of the
    same misfit (hf_calib_run) and a plain solve of the same steps (hf_sim
    run_steps); checked against the Dual tangent in 8 seeded Gaussian
    directions and against central differences (eps = 1e-6, dt frozen).
    Replicas on N > 1 (each rank its own copy; max over ranks)."""
    import torch

    from hydroflux_b200 import _lib, calib, workloads
    dev = d.local
    torch.cuda.set_device(dev)
    _lib.lib()
    P = workloads.calibration_problem(n=a.calib_n, n_steps=a.calib_steps)
    s = P.scenario
    K = P.n_steps
    reps = min(max(a.steps, 1), 5)  # each repetition is a full forward + gradient
    with calib.Calibration(s, K, P.gauges, checkpoint_every=a.checkpoint_every,
                           device=dev) as cal:
        _, gh, k_obs = cal.run(P.manning_true)
        obs = np.zeros((K, len(P.gauges)))
        obs[:k_obs] = gh
        cal.set_observations(obs)
        for _ in range(max(a.warmup, 3) if a.warmup else 1):
            cal.run(s.manning)
            cal.gradient(s.manning)
        torch.cuda.synchronize(dev)
        d.barrier()
        clocks = ClockSampler(dev)
        clocks.start()
        t_fwd, t_grad = [], []
        k_launch = launches()
        for _ in range(reps):
            t0 = time.perf_counter()
            J, _, k_run = cal.run(s.manning)
            t1 = time.perf_counter()
            Jg, g = cal.gradient(s.manning)
            t2 = time.perf_counter()
            t_fwd.append(t1 - t0)
            t_grad.append(t2 - t1)
        k_launch = (launches() - k_launch) // max(reps, 1)
        clk = clocks.stop()
        f_s = d.max(statistics.median(t_fwd))
        g_s = d.max(statistics.median(t_grad))
        # checks: Dual tangent in 8 directions, central differences in 2
        rng = np.random.default_rng(12345)
        dot_errs, t_tan = [], []
        for _ in range(8):
            v = rng.standard_normal(s.shape) * s.manning * 0.01
            t0 = time.perf_counter()
            _, dJ = cal.tangent(s.manning, dn=v)
            t_tan.append(time.perf_counter() - t0)
            ad = float(np.sum(g * v))
            dot_errs.append(abs(ad - dJ) / max(abs(dJ), 1e-300))
        fd_errs = []
        cal.run(s.manning)  # dt record of the base field
        for _ in range(2):
            v = rng.standard_normal(s.shape) * s.manning
            eps = 1e-6
            Jp, _, _ = cal.run(s.manning + eps * v, replay_dt=True)
            Jm, _, _ = cal.run(s.manning - eps * v, replay_dt=True)
            fd = (Jp - Jm) / (2 * eps)
            ad = float(np.sum(g * v))
            fd_errs.append({"fd": fd, "adjoint": ad, "rel": abs(fd - ad) / max(abs(ad), 1e-300)})
    with workloads.simulation_for(s, device=dev) as sm:
        sm.run_steps(3, s.t_end)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        sm.run_steps(K, s.t_end)
        torch.cuda.synchronize(dev)
        plain_s = d.max(time.perf_counter() - t0)
    # Where the linearization stops predicting: adjoint vs central differences
    # and the size of the tangent state, by misfit horizon.
    by_horizon = []
    for Kh in (h for h in (50, 100, 200, 500, 1000, 2000) if h <= K):
        Ph = workloads.calibration_problem(n=a.calib_n, n_steps=Kh)
        with calib.Calibration(Ph.scenario, Kh, Ph.gauges, checkpoint_every=a.checkpoint_every,
                               device=dev) as ch:
            _, gh, ko = ch.run(Ph.manning_true)
            ob = np.zeros((Kh, len(Ph.gauges)))
            ob[:ko] = gh
            ch.set_observations(ob)
            Jh, gg = ch.gradient(Ph.scenario.manning)
            rr = np.random.default_rng(777)
            v = rr.standard_normal(Ph.scenario.shape) * Ph.scenario.manning
            ad = float(np.sum(gg * v))
            ch.run(Ph.scenario.manning)
            eps = 1e-6
            Jp, _, _ = ch.run(Ph.scenario.manning + eps * v, replay_dt=True)
            Jm, _, _ = ch.run(Ph.scenario.manning - eps * v, replay_dt=True)
            fd = (Jp - Jm) / (2 * eps)
            ch.tangent(Ph.scenario.manning, dn=v)
            st = ch.final_state()
            by_horizon.append({"steps": Kh, "J": Jh, "adjoint": ad, "fd": fd,
                               "rel": abs(fd - ad) / max(abs(ad), 1e-300),
                               "max_abs_dh": float(np.max(np.abs(st["dh"])))})
    ncell = s.n_cells
    line = {"metric": "misfit gradient time / forward solve time", "value": g_s / f_s,
            "unit": "x", "n_gpus": d.world, "steps": reps, "warmup": max(a.warmup, 3),
            "higher_is_better": False, "scaling": "replicas",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded valley, log-normal Manning field, hidden-field gauges)",
            "config": {"workload": f"Manning-field gradient of a 16-gauge misfit over {K} steps, "
                                   f"valley {a.calib_n}x{a.calib_n}, dx 5 m, log-normal n "
                                   "(median 0.04, sigma 0.3, 10-cell smoothing)",
                       "cells": ncell, "misfit_steps": int(k_run),
                       "checkpoint_every": a.checkpoint_every, "parallelism": "replicas"},
            "gradient_s": g_s, "forward_s": f_s, "plain_solve_s": plain_s,
            "gradient_vs_plain_solve": g_s / plain_s,
            "tangent_s": statistics.median(t_tan), "J": Jg,
            "checks": {"dual_tangent_8_dirs_max_rel": max(dot_errs),
                       "central_fd_eps1e-6": fd_errs, "fd_by_horizon": by_horizon},
            # per misfit step: primal 5, replay 3, reverse 7 launches
            "gpu_launches": k_launch, "gpu_launches_per": "one forward solve + one gradient",
            "clocks": clk}
    if d.rank == 0:
        print(json.dumps(line), flush=True)


def run_lanes(a, d: Dist):
    """Forward-mode gradients for P zonal Manning parameters (vertical
    stripes), the trade-off of solver-2d/examples/m1_forward_scaling.rs: P
    scalar Dual runs (hf_tangent) against one vector-mode run with P lanes
    (hf_tangent_lanes) and against one reverse sweep (hf_grad_manning), each
    as a multiple of the forward misfit solve. On the misfit problem of the
    adjoint line (--calib-n, --calib-steps) and on a 64x64 grid of the same
    generator, where one Dual grid fills only a tenth of the SMs. Lane
    derivatives are checked against the zone sums of the adjoint gradient.
    Replicas on N > 1."""
    import torch

    from hydroflux_b200 import _lib, calib, workloads
    dev = d.local
    torch.cuda.set_device(dev)
    _lib.lib()
    counts = (1, 2, 4, 8, 16)
    by_grid = {}
    t_all = 0.0
    clocks = ClockSampler(dev)
    clocks.start()
    for n_side in (a.calib_n, 64):
        P = workloads.calibration_problem(n=n_side, n_steps=a.calib_steps)
        s = P.scenario
        K = P.n_steps
        with calib.Calibration(s, K, P.gauges, device=dev) as cal:
            _, gh, k_obs = cal.run(P.manning_true)
            obs = np.zeros((K, len(P.gauges)))
            obs[:k_obs] = gh
            cal.set_observations(obs)
            cols = np.arange(s.shape[1])
            for _ in range(max(a.warmup, 3)):
                cal.run(s.manning)
            cal.tangent(s.manning, dn=np.ones(s.shape))  # captures the tangent's graphs
            cal.gradient(s.manning)  # allocates the adjoint's buffers
            torch.cuda.synchronize(dev)

            def timed(fn):
                timed.k = launches()
                t0 = time.perf_counter()
                out = fn()
                torch.cuda.synchronize(dev)
                el = time.perf_counter() - t0
                timed.k = launches() - timed.k
                return el, out

            f_s, _ = timed(lambda: cal.run(s.manning))
            g_s, (_, g) = timed(lambda: cal.gradient(s.manning))
            rows = []
            for Pn in counts:
                zone = (cols * Pn) // s.shape[1]
                dn = np.stack([np.broadcast_to((zone == p).astype(float), s.shape)
                               for p in range(Pn)])
                sc_s, sc = timed(lambda: [cal.tangent(s.manning, dn=dn[p])[1] for p in range(Pn)])
                # untimed first call at this lane count: lane buffers and graphs
                cal.tangent_lanes(s.manning, dn=dn)
                vm_s, (_, dJ) = timed(lambda: cal.tangent_lanes(s.manning, dn=dn))
                vm_k = timed.k
                same = bool(np.array_equal(np.array(sc), dJ))
                zs = np.array([np.sum(g[:, zone == p]) for p in range(Pn)])
                rel = float(np.max(np.abs(zs - dJ) / np.maximum(np.abs(dJ), 1e-300)))
                rows.append({"P": Pn, "scalar_s": d.max(sc_s), "vector_s": d.max(vm_s),
                             "scalar_vs_forward": d.max(sc_s) / d.max(f_s),
                             "vector_vs_forward": d.max(vm_s) / d.max(f_s),
                             "vector_per_param": (d.max(vm_s) / d.max(f_s)) / Pn,
                             "lanes_equal_scalar_runs": same, "vector_gpu_launches": vm_k,
                             "adjoint_zone_sums_max_rel": rel})
                t_all += sc_s + vm_s
        by_grid[f"{n_side}x{n_side}"] = {"cells": s.n_cells, "misfit_steps": K,
                                         "forward_s": d.max(f_s), "gradient_s": d.max(g_s),
                                         "gradient_vs_forward": d.max(g_s) / d.max(f_s),
                                         "rows": rows}
    clk = clocks.stop()
    main_rows = by_grid[f"{a.calib_n}x{a.calib_n}"]["rows"]
    p16 = [r for r in main_rows if r["P"] == 16][0]
    line = {"metric": "16-parameter forward-mode gradient time / forward solve time (vector mode)",
            "value": p16["vector_vs_forward"], "unit": "x", "n_gpus": d.world,
            "steps": len(counts), "warmup": max(a.warmup, 3), "higher_is_better": False,
            "scaling": "replicas", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded valley, log-normal Manning field, hidden-field gauges)",
            "config": {"workload": f"zonal Manning derivatives (P vertical stripes) of a 16-gauge "
                                   f"misfit over {a.calib_steps} steps, valley {a.calib_n}x"
                                   f"{a.calib_n} and 64x64, dx 5 m",
                       "parallelism": "replicas"},
            "by_grid": by_grid,
            "note": "steady state: each lane count runs once untimed (lane buffers, graph "
                    "capture) before its timed run; the scalar tangent's graphs are captured "
                    "in the warm-up",
            "gpu_launches": p16["vector_gpu_launches"], "clocks": clk}
    if d.rank == 0:
        print(json.dumps(line), flush=True)


def run_serve(a, d: Dist):
    """An arrival stream through the continuous-batching server (hf_server_*)
    against a sequential plain solve per request (hf_sim run_until, FIFO, one
    at a time, same requests): p50/p99 latency (arrival -> result) and
    solves/s. The sequential server's latencies come from the measured
    per-request solve times queued in arrival order. The stream is split over
    ranks by work (cells x horizon, longest first to the lightest rank); rank
    0 gathers every request's latency."""
    import torch

    from hydroflux_b200 import _lib, serve, workloads
    dev = d.local
    torch.cuda.set_device(dev)
    _lib.lib()
    sides = tuple(int(x) for x in a.sides.split(","))
    h0, h1 = (float(x) for x in a.horizon.split(","))
    reqs = serve.request_stream(a.requests, rate=a.rate, seed=7, sides=sides, horizon_min=h0,
                                horizon_max=h1, max_dt=60.0)
    t_gen = time.perf_counter()
    for r in reqs:  # payloads (bed, n, forcings) arrive with the request
        r.prepare()
    gen_s = time.perf_counter() - t_gen
    mine = [reqs[i] for i in d.shard([r.work() for r in reqs])]
    # warm-up: one small request through each path
    warm = serve.request_stream(2, rate=1e6, seed=99, sides=(64,), horizon_min=5.0,
                                horizon_max=10.0)
    serve.serve_stream(warm, hbm_budget_bytes=150 << 30, device=dev)
    torch.cuda.synchronize(dev)
    d.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    k_serve = launches()
    out = serve.serve_stream(mine, hbm_budget_bytes=150 << 30, device=dev, policy="srpt",
                             max_active_cells=a.max_active_cells)
    k_serve = launches() - k_serve
    clk = clocks.stop()
    fifo = {"latencies": [], "makespan": float("nan")}
    if not a.no_fifo:
        for r in mine:
            r.admitted = r.done = r.result = None
        fifo = serve.serve_stream(mine, hbm_budget_bytes=150 << 30, device=dev, policy="fifo")
    # sequential plain solves in arrival order
    ordered = sorted(mine, key=lambda q: q.arrival)
    service = []
    for r in ordered:
        s = r.prepare()
        with workloads.simulation_for(s, device=dev) as sm:
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            sm.run_until(s.t_end)
            torch.cuda.synchronize(dev)
            service.append(time.perf_counter() - t0)
    t_free, lat = 0.0, []
    for r, sv in zip(ordered, service):
        start = max(r.arrival, t_free)
        t_free = start + sv
        lat.append(t_free - r.arrival)
    # whole-job figures: latencies of every rank's requests, the slowest rank's makespan
    per_rank = d.gather({"served": list(out["latencies"]),
                         "fifo": list(fifo["latencies"]), "seq": lat,
                         "makespan": out["makespan"], "fifo_makespan": fifo["makespan"],
                         "seq_end": t_free, "busy": float(sum(service)), "k": k_serve})
    if d.rank != 0:
        return
    cat = lambda k: np.concatenate([np.asarray(x[k], dtype=np.float64) for x in per_rank])  # noqa: E731
    n_all = len(cat("served"))
    mk = max(x["makespan"] for x in per_rank)
    out = {"latency_p50": float(np.percentile(cat("served"), 50)),
           "latency_p99": float(np.percentile(cat("served"), 99)),
           "solves_per_s": n_all / mk, "makespan": mk, "failed": out["failed"]}
    fmk = max(x["fifo_makespan"] for x in per_rank)
    fifo = {"latency_p50": float(np.percentile(cat("fifo"), 50)) if not a.no_fifo else None,
            "latency_p99": float(np.percentile(cat("fifo"), 99)) if not a.no_fifo else None,
            "solves_per_s": n_all / fmk if not a.no_fifo else None, "makespan": fmk}
    seq_end = max(x["seq_end"] for x in per_rank)
    seq = {"latency_p50": float(np.percentile(cat("seq"), 50)),
           "latency_p99": float(np.percentile(cat("seq"), 99)),
           "solves_per_s": n_all / seq_end, "busy_s": float(sum(x["busy"] for x in per_rank)),
           "latencies": "each request's plain solve time measured alone, then queued in "
                        "arrival order (FIFO, one at a time); not a live stream"}
    line = {"metric": "served solves/s", "value": out["solves_per_s"],
            "unit": "solves/s", "n_gpus": d.world, "steps": n_all, "warmup": 2,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded valley per request)",
            "config": {"workload": f"Poisson stream, {a.requests} requests at {a.rate}/s, side "
                                   f"uniform over {list(sides)}, horizon U[{h0}, {h1}] s, valley "
                                   "DEM / n / inflow per request seed, HBM budget 150 GB",
                       "parallelism": f"requests sharded over {d.world} GPU(s) by work"},
            "latency_p50_s": out["latency_p50"], "latency_p99_s": out["latency_p99"],
            "failed": out["failed"], "makespan_s": out["makespan"],
            "admission": f"shortest work (cells x horizon) first, at most "
                         f"{a.max_active_cells} cells advancing together",
            "fifo_uncapped": {k: fifo[k] for k in ("latency_p50", "latency_p99",
                                                   "solves_per_s", "makespan")},
            "payload_generation_s": gen_s,
            "sequential_plain": seq,
            "speedup_solves_per_s": out["solves_per_s"] / seq["solves_per_s"],
            "gpu_launches": sum(x["k"] for x in per_rank), "clocks": clk}
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    d = Dist(use_gpu=a.impl == "ours")
    try:
        if a.impl == "reference":
            run_reference(a, d)
        elif a.workload == "ensemble":
            run_ensemble(a, d)
        elif a.workload == "adjoint":
            run_adjoint(a, d)
        elif a.workload == "serve":
            run_serve(a, d)
        elif a.workload == "lanes":
            run_lanes(a, d)
        elif a.workload == "regimes":
            run_regimes(a, d)
        else:
            run_ours(a, d)
    finally:
        d.close()


if __name__ == "__main__":
    main()
