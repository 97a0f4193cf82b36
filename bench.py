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
    p.add_argument("--workload", default="valley", choices=["valley", "ensemble"],
                   help="valley: the 4096^2 plain step (default line); ensemble: batched "
                        "uneven-size scenarios vs a loop of per-scenario solves")
    p.add_argument("--scenarios", type=int, default=512)
    p.add_argument("--loop-every", type=int, default=8,
                   help="ensemble: the per-scenario loop times every k-th scenario")
    p.add_argument("--complete", action="store_true",
                   help="ensemble: also run the batch to every scenario's horizon")
    return p.parse_args()


# --------------------------------------------------------------------- dist
class Dist:
    def __init__(self, use_gpu: bool):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        if self.world > 1 and use_gpu:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", self.local))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


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


def profiled_traffic():
    """DRAM bytes per stage launch per cell from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "stage_kernel_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_cell_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------- workload
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
def run_ours(a, d: Dist):
    import torch

    from hydroflux_b200 import _lib, workloads
    dev = d.local
    torch.cuda.set_device(dev)
    _lib.lib()
    scn = make_workload(a.n)
    cells = scn.n_cells

    sm = workloads.simulation_for(scn, device=dev)
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
    sm.run_steps(a.steps, scn.t_end)
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
    traffic_per_cell = profiled_traffic()
    sm.close()

    # ---- e2e: through the C ABI with host buffers (pinned), copies timed
    e2e = None
    if not a.no_e2e:
        from hydroflux_b200 import sim as S
        scn_w = scn
        bed_p = torch.from_numpy(scn.bed).pin_memory()
        man_p = torch.from_numpy(scn.manning).pin_memory()
        torch.cuda.synchronize(dev)
        d.barrier()
        t_a = time.perf_counter()
        cfg = S.SimulationConfig(cfl=scn_w.cfl, boundaries=S.Boundaries2D(
            *[S.Boundary(k, v) for k, v in scn_w.bcs]), max_dt=scn_w.max_dt)
        mesh = S.Mesh2D(bed_p.numpy(), scn_w.dx, scn_w.dy, man_p.numpy())
        st = tuple(p_.numpy() for p_ in pinned)
        s2 = S.Simulation(mesh, st, cfg, dev)
        s2.set_rain(np.stack(scn_w.rain, axis=1))
        s2.set_point_sources([S.PointSource(r, c, np.stack([t, q], axis=1))
                              for r, c, t, q in scn_w.sources])
        for _ in range(a.steps):
            s2.step(scn_w.t_end - s2.time())
        out = [torch.empty(scn.shape, dtype=torch.float64, pin_memory=True) for _ in range(3)]
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
               "note": "Simulation::new from pinned host arrays (bed, n, h, hu, hv), K x "
                       "Simulation::step through the C ABI (dt read back each step), "
                       "states() to pinned host; copies, allocation and graph capture timed"}

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
        "config": {"workload": f"valley flood {a.n}x{a.n}, dx=5 m, SSP-RK2 + Manning + rain + "
                               f"point inflow, CFL 0.5, transmissive sides",
                   "grid": f"{a.n}x{a.n}", "cells": cells, "integrator": "ssprk2",
                   "wet_fraction": round(wet_frac, 4),
                   "l2": "inputs larger than L2 (h,hu,hv,z,n = 40 B/cell resident)",
                   "parallelism": f"replicas x{d.world}" if d.world > 1 else "single grid"},
        "e2e": e2e,
        "gpu_launches": 3 * a.steps,
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                     "frac": achieved_gbs / peak, "peak_source": peak_kind,
                     "traffic": (traffic_per_cell * cells) if traffic_per_cell else None,
                     "kernel": "k_stage", "alg_bytes_per_launch": bytes_per_launch,
                     "avg_launch_ms": avg_stage_s * 1e3, "launches": stage_launches},
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    if d.rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------ reference arm (CPU)
def run_reference(a, d: Dist):
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
    # Warm-up: the first steps wet the dry valley (rain), as in the GPU arm.
    warm = min(max(a.warmup, 1), 2)
    r = O.sim_run(scn.bed, scn.manning, scn.dx, scn.dy, scn.h, scn.hu, scn.hv, cfg, scn.t_end,
                  forcing=f, stop_after=warm)
    t0 = time.perf_counter()
    r1 = O.sim_run(scn.bed, scn.manning, scn.dx, scn.dy, r["h"], r["hu"], r["hv"], cfg, scn.t_end,
                   forcing=f, stop_after=1, t0=r["t"], steps0=r["steps"])
    per_step = time.perf_counter() - t0
    budget_s = 150.0
    k = max(1, min(a.steps, int(budget_s / max(per_step, 1e-3))))
    t0 = time.perf_counter()
    r2 = O.sim_run(scn.bed, scn.manning, scn.dx, scn.dy, r1["h"], r1["hu"], r1["hv"], cfg,
                   scn.t_end, forcing=f, stop_after=k, t0=r1["t"], steps0=r1["steps"])
    el = time.perf_counter() - t0
    assert r2["status"] == 0, r2["message"]
    value = cells * k / el
    sample = (f"{k} of the requested {a.steps} steps on the full {a.n}^2 workload after "
              f"{warm + 1} warm-up steps; CPU oracle (C++ restatement of the reference, "
              f"OpenMP row chunks like its rayon feature), {threads} threads")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": k,
            "warmup": warm + 1, "ms_per_step": el / k * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded valley DEM, Voronoi Manning field, rain + inflow hydrograph)",
            "config": {"workload": f"valley flood {a.n}x{a.n}, dx=5 m, SSP-RK2 + Manning + rain "
                                   f"+ point inflow, CFL 0.5, transmissive sides",
                       "grid": f"{a.n}x{a.n}", "cells": cells, "integrator": "ssprk2"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ensemble(a, d: Dist):
    """Batched ensemble (hf_batch_*) against a loop of per-scenario plain GPU
    solves (hf_sim run_steps, one scenario after another), same scenarios and
    the same number of steps per scenario. Scenarios are sharded over ranks
    (every world-th scenario per rank; no collective)."""
    import torch

    from hydroflux_b200 import _lib, workloads
    from hydroflux_b200.ensemble import Ensemble, ensemble_scenarios
    dev = d.local
    torch.cuda.set_device(dev)
    _lib.lib()
    t_gen = time.perf_counter()
    allscn = ensemble_scenarios(count=a.scenarios, seed=0)
    mine = allscn[d.rank::d.world]
    gen_s = time.perf_counter() - t_gen
    cells = np.array([s.n_cells for s in mine], dtype=np.float64)
    ens = Ensemble(mine, device=dev)
    ens.run(max(a.warmup, 3))
    st0 = np.array([ens.info(k)["steps"] for k in range(len(mine))], dtype=np.float64)
    torch.cuda.synchronize(dev)
    d.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    t0 = time.perf_counter()
    left = ens.run(a.steps)
    t1 = time.perf_counter()
    clk = clocks.stop()
    st1 = np.array([ens.info(k)["steps"] for k in range(len(mine))], dtype=np.float64)
    el = d.max(t1 - t0)
    batched = float(np.sum(cells * (st1 - st0)))
    batched_rate = d.world * batched / el
    complete = None
    if a.complete:
        t2 = time.perf_counter()
        left = ens.run()
        t3 = time.perf_counter()
        done = sum(1 for k in range(len(mine)) if ens.info(k)["status"] == 0)
        complete = {"seconds": t3 - t2 + (t1 - t0), "scenarios_completed": done,
                    "solves_per_s": done / (t3 - t2 + (t1 - t0)), "unfinished": left}
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
            "warmup": max(a.warmup, 3), "higher_is_better": True, "scaling": "weak",
            "dtype": "f64", "data": "synthetic (seeded valley ensemble)",
            "config": {"workload": f"{a.scenarios} scenarios, side log-uniform in [64, 1024], "
                                   "valley DEM per-scenario seed, n ~ U[0.02, 0.08], inflow "
                                   "peak 500 x U[0.5, 2] m^3/s, horizon 30 min, dx 5 m",
                       "cells": int(sum(s.n_cells for s in allscn)),
                       "parallelism": f"scenarios sharded over {d.world} GPU(s)"},
            "loop_of_plain_solves": {"value": loop_rate, "unit": "cell-updates/s",
                                     "scenarios_timed": len(sub)},
            "speedup_vs_loop": (batched_rate / d.world) / loop_rate if loop_rate else None,
            "gpu_launches": 4 * a.steps, "generation_s": gen_s, "complete": complete,
            "clocks": clk}
    if d.rank == 0:
        print(json.dumps(line), flush=True)


def main():
    a = parse()
    d = Dist(use_gpu=a.impl == "ours")
    try:
        if a.impl == "reference":
            run_reference(a, d)
        elif a.workload == "ensemble":
            run_ensemble(a, d)
        else:
            run_ours(a, d)
    finally:
        d.close()


if __name__ == "__main__":
    main()
