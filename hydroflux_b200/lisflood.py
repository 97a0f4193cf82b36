"""LISFLOOD-FP benchmark inputs driven through the B200 solver.

The reference validates its solver on real terrain with the UK Environment
Agency 2D benchmarks, distributed as LISFLOOD-FP input decks: a parameter
file (.par), ESRI ASCII DEM and roughness grids, boundary conditions
(.bci / .bdy), a hyetograph (.rain) and control points (.stage). Its
examples (solver-2d/examples/uk_ea_test4_official.rs,
uk_ea_test8a_official.rs) hard-code the decks' tables; this module reads the
decks and builds the same run:

- point inflow `P x y QVAR name`: one PointSource at cell_at(x, y) with
  q = QVAR(t) * cellsize (uk_ea_test8a_official.rs:131-134, 207-214);
- line inflow `W|E lo hi QVAR name`: one PointSource per row overlapping
  [lo, hi) at the edge column, q = (QVAR(t) * (hi - lo)) / rows; that side
  stays a wall (uk_ea_test4_official.rs:107-118, 183-195);
- `N|S|E|W ... FREE`: a transmissive side; unlisted sides are walls;
- rain: the .rain hyetograph in mm/h, rate = (v * 1e-3) / 3600
  (uk_ea_test8a_official.rs:126-129);
- each series evaluated at t_new after every step, in the file's time unit
  (t / 60 for minutes), the rain first (ibid. 203-217).

The series units, the forcing order and the control-point recording run on
the device (Simulation.set_rain_units, set_point_source_units, set_gauges),
so a whole event is one run_until call. `read_reference_stage`,
`interp` and `compare_point` restate the examples' comparison against
LISFLOOD-FP output (solver-2d/examples/uk_ea_common/mod.rs:47-190).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import raster
from .sim import (Boundaries2D, Boundary, PointSource, Simulation, SimulationConfig)

UNIT_SECONDS = {"seconds": 1.0, "minutes": 60.0, "hours": 3600.0}


def _text_lines(path) -> List[str]:
    with open(path, "r", encoding="utf-8") as f:
        return [ln.rstrip("\r\n").rstrip("\r") for ln in f.read().split("\n")]


def _resolve(base_dir: str, name: str) -> str:
    """A deck file name, or its .gz when only that is shipped."""
    p = name if os.path.isabs(name) else os.path.join(base_dir, name)
    if os.path.exists(p):
        return p
    if os.path.exists(p + ".gz"):
        return p + ".gz"
    raise FileNotFoundError(p)


def read_par(path) -> Dict[str, object]:
    """`key value` lines; a key alone is a flag (True); '#' starts a comment."""
    out: Dict[str, object] = {}
    for ln in _text_lines(path):
        toks = ln.split("#", 1)[0].split()
        if not toks:
            continue
        out[toks[0]] = toks[1] if len(toks) > 1 else True
    return out


def read_stage_points(path) -> List[Tuple[float, float]]:
    """Control points: a count, then `x y` per line."""
    lines = [ln.split() for ln in _text_lines(path) if ln.strip()]
    n = int(lines[0][0])
    return [(float(t[0]), float(t[1])) for t in lines[1:1 + n]]


@dataclass
class BciEntry:
    kind: str             # 'P' (point) or a side 'N' / 'S' / 'E' / 'W'
    a: float              # point x, or the start of the side's segment
    b: float              # point y, or the end of the segment
    bctype: str           # QVAR, FREE, ...
    value: Optional[str]  # series name (QVAR) or constant


def read_bci(path) -> List[BciEntry]:
    out = []
    for ln in _text_lines(path):
        toks = ln.split()
        if len(toks) < 4:
            continue
        out.append(BciEntry(toks[0].upper(), float(toks[1]), float(toks[2]), toks[3].upper(),
                            toks[4] if len(toks) > 4 else None))
    return out


def _series_block(lines: List[List[str]], i: int):
    n, unit = int(float(lines[i][0])), lines[i][1].lower()
    rows = lines[i + 1:i + 1 + n]
    v = np.array([float(r[0]) for r in rows])
    t = np.array([float(r[1]) for r in rows])
    return t, v, unit, i + 1 + n


def read_bdy(path) -> Dict[str, Tuple[np.ndarray, np.ndarray, str]]:
    """Named series: a comment line, then blocks of `name`, `n unit` and n
    `value time` rows. Returns name -> (t in the file's unit, value, unit)."""
    lines = [ln.split() for ln in _text_lines(path)[1:] if ln.strip()]
    out, i = {}, 0
    while i < len(lines):
        name = lines[i][0]
        t, v, unit, i = _series_block(lines, i + 1)
        out[name] = (t, v, unit)
    return out


def read_rain(path) -> Tuple[np.ndarray, np.ndarray, str]:
    """A comment line, `n unit`, then n `value time` rows (value in mm/h)."""
    lines = [ln.split() for ln in _text_lines(path)[1:] if ln.strip()]
    t, v, unit, _ = _series_block(lines, 0)
    return t, v, unit


@dataclass
class ReferenceStage:
    """ReferenceStage (uk_ea_common/mod.rs:22-31)."""
    points: List[Tuple[float, float]]
    times: np.ndarray
    depths: np.ndarray  # (len(times), len(points))


def _f64_or_none(tok: str):
    try:
        return float(tok)
    except ValueError:
        return None


def read_reference_stage(path) -> ReferenceStage:
    """parse_reference_stage (uk_ea_common/mod.rs:47-106): the coordinate
    block after the `stage,x,y,elev` marker, then `time depth...` rows
    after the `Time;` header (rows of the wrong width are skipped)."""
    lines = _text_lines(path)
    i = 0
    while i < len(lines) and "stage,x,y,elev" not in lines[i]:
        i += 1
    i += 1
    points = []
    while i < len(lines):
        toks = lines[i].split()
        i += 1
        if len(toks) < 3:
            break
        x, y = _f64_or_none(toks[1]), _f64_or_none(toks[2])
        if x is None or y is None:
            break
        points.append((x, y))
    while i < len(lines):
        i += 1
        if "Time;" in lines[i - 1]:
            break
    times, depths = [], []
    for ln in lines[i:]:
        vals = [_f64_or_none(t) for t in ln.split()]
        if any(v is None for v in vals) or len(vals) != len(points) + 1:
            continue
        times.append(vals[0])
        depths.append(vals[1:])
    if not points or not times:
        raise ValueError(f"no control points or data rows parsed from {path}")
    return ReferenceStage(points, np.array(times), np.array(depths))


def interp(times: Sequence[float], values: Sequence[float], t: float) -> float:
    """interp (uk_ea_common/mod.rs:108-120): piecewise linear, clamped."""
    if t <= times[0]:
        return float(values[0])
    if t >= times[-1]:
        return float(values[-1])
    idx = int(np.searchsorted(np.asarray(times), t, side="right"))  # partition_point(ti <= t)
    t0, t1 = times[idx - 1], times[idx]
    v0, v1 = values[idx - 1], values[idx]
    frac = (t - t0) / (t1 - t0)
    return float(v0 + frac * (v1 - v0))


@dataclass
class PointComparison:
    rmse: float
    peak_bias: float
    reference_peak: float
    reference_arrival: Optional[float]
    sim_arrival: Optional[float]


def _arrival(times, values, threshold):
    for t, v in zip(times, values):
        if v > threshold:
            return float(t)
    return None


def compare_point(reference: ReferenceStage, p: int, sim_times, sim_values,
                  arrival_threshold: float) -> PointComparison:
    """compare_point (uk_ea_common/mod.rs:163-190): the simulated series
    interpolated onto the reference's times; RMSE, peak bias (peaks are
    fold(0.0, f64::max)) and first times above the threshold."""
    ref = reference.depths[:, p]
    sim = [interp(sim_times, sim_values, t) for t in reference.times]
    mse = 0.0
    for r, s in zip(ref, sim):
        mse += (r - s) ** 2
    mse /= len(ref)
    ref_peak = 0.0
    for r in ref:
        ref_peak = max(ref_peak, r) if r == r else ref_peak
    sim_peak = 0.0
    for s in sim:
        sim_peak = max(sim_peak, s) if s == s else sim_peak
    return PointComparison(math.sqrt(mse), sim_peak - ref_peak, ref_peak,
                           _arrival(reference.times, ref, arrival_threshold),
                           _arrival(reference.times, sim, arrival_threshold))


@dataclass
class Case:
    """One LISFLOOD-FP deck as a solver run."""
    mesh: object
    header: raster.AsciiGridHeader
    config: SimulationConfig
    sim_time: float
    points: List[Tuple[float, float]]
    gauges: List[Tuple[int, int]]
    rain: Optional[Tuple[np.ndarray, np.ndarray]] = None
    rain_units: Tuple[float, float, float] = (1.0, 1.0, 1.0)
    sources: List[Tuple[int, int, np.ndarray, np.ndarray]] = field(default_factory=list)
    source_units: Tuple[float, float, float] = (1.0, 1.0, 1.0)

    def forcing_series(self):
        """(rain, sources) as plain (t, v) arrays, for the oracle."""
        return self.rain, self.sources


def load_case(par_path, dem: Optional[str] = None, cfl: float = 0.4,
              max_dt: float = 60.0) -> Case:
    """Build the run of a LISFLOOD-FP deck. `dem` overrides the .par's
    DEMfile (the decks ship several resolutions); `cfl` and `max_dt` are the
    solver settings the reference examples choose (0.4, and 15 s / 10 s as
    the dry-start cap: uk_ea_test4_official.rs:131-146,
    uk_ea_test8a_official.rs:174-183)."""
    base = os.path.dirname(os.path.abspath(par_path))
    par = read_par(par_path)
    dem_path = _resolve(base, dem or str(par["DEMfile"]))
    if "manningfile" in par:
        mesh, header = raster.mesh_from_ascii_grid(dem_path,
                                                   _resolve(base, str(par["manningfile"])))
    elif "fpfric" in par:
        mesh, header = raster.mesh_from_ascii_grid(dem_path, float(par["fpfric"]))
    else:
        raise ValueError("the deck sets neither manningfile nor fpfric")
    if not np.all(np.isfinite(mesh.bed)) or np.any(mesh.bed == header.nodata_value):
        raise ValueError("the DEM has NODATA cells; masked cells are not supported")
    sides = {"N": Boundary.wall(), "S": Boundary.wall(), "W": Boundary.wall(),
             "E": Boundary.wall()}
    bdy = read_bdy(_resolve(base, str(par["bdyfile"]))) if "bdyfile" in par else {}
    sources, units = [], None
    cs = header.cellsize

    def add_units(u):
        nonlocal units
        if units is not None and units != u:
            raise NotImplementedError("point sources with different series units")
        units = u

    for e in (read_bci(_resolve(base, str(par["bcifile"]))) if "bcifile" in par else []):
        if e.bctype == "FREE" and e.kind in sides:
            sides[e.kind] = Boundary.transmissive()
        elif e.bctype == "QVAR" and e.kind == "P":
            t, v, unit = bdy[e.value]
            cell = header.cell_at(e.a, e.b)
            if cell is None:
                raise ValueError(f"point inflow ({e.a}, {e.b}) is outside the grid")
            sources.append((cell[0], cell[1], t, v))
            add_units((UNIT_SECONDS[unit], cs, 1.0))
        elif e.bctype == "QVAR" and e.kind in ("W", "E"):
            t, v, unit = bdy[e.value]
            rows = header.rows_overlapping_y_range(e.a, e.b)
            if not rows:
                raise ValueError(f"inflow segment [{e.a}, {e.b}) is outside the grid")
            col = 0 if e.kind == "W" else header.ncols - 1
            for r in rows:
                sources.append((r, col, t, v))
            add_units((UNIT_SECONDS[unit], e.b - e.a, float(len(rows))))
        else:
            raise NotImplementedError(f"boundary condition {e.kind} {e.bctype}")
    bcs = Boundaries2D(north=sides["N"], south=sides["S"], west=sides["W"], east=sides["E"])
    config = SimulationConfig(cfl=cfl, boundaries=bcs, max_dt=max_dt)
    rain, rain_units = None, (1.0, 1.0, 1.0)
    if "rainfall" in par:
        t, v, unit = read_rain(_resolve(base, str(par["rainfall"])))
        rain, rain_units = (t, v), (UNIT_SECONDS[unit], 1e-3, 3600.0)
    points = read_stage_points(_resolve(base, str(par["stagefile"])))
    gauges = []
    for x, y in points:
        c = header.cell_at(x, y)
        if c is None:
            raise ValueError(f"control point ({x}, {y}) is outside the grid")
        gauges.append(c)
    return Case(mesh, header, config, float(par["sim_time"]), points, gauges, rain, rain_units,
                sources, units or (1.0, 1.0, 1.0))


def simulation(case: Case, device: int = 0, capacity: int = 1 << 20) -> Simulation:
    """The deck's Simulation: dry start, forcings, control points."""
    shape = case.mesh.bed.shape
    zero = np.zeros(shape)
    sim = Simulation(case.mesh, (zero, zero, zero), case.config, device)
    if case.rain is not None:
        sim.set_rain(np.stack(case.rain, axis=1))
        sim.set_rain_units(*case.rain_units)
    if case.sources:
        sim.set_point_sources([PointSource(r, c, np.stack((t, v), axis=1))
                               for r, c, t, v in case.sources])
        sim.set_point_source_units(*case.source_units)
    sim.set_gauges(case.gauges, capacity)
    return sim


def run_case(case: Case, device: int = 0, capacity: int = 1 << 20) -> dict:
    """The whole event in one run_until; host wall time around it."""
    sim = simulation(case, device, capacity)
    t0 = time.perf_counter()
    sim.run_until(case.sim_time)
    wall = time.perf_counter() - t0
    peaks, finals = sim.gauge_peaks()
    times, depths, seen = sim.gauge_series()
    out = dict(steps=sim.steps(), t=sim.time(), wall_s=wall, peaks=peaks, finals=finals,
               times=times, depths=depths, rows_seen=seen, state=sim.states())
    sim.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description="Run a LISFLOOD-FP deck on the B200 solver.")
    ap.add_argument("par")
    ap.add_argument("--dem", default=None, help="DEM file name overriding the .par's DEMfile")
    ap.add_argument("--max-dt", type=float, default=60.0)
    ap.add_argument("--cfl", type=float, default=0.4)
    ap.add_argument("--reference-stage", nargs="*", default=[],
                    help="LISFLOOD-FP .stage output files to compare against")
    ap.add_argument("--arrival-threshold", type=float, default=0.02)
    ap.add_argument("--json", default=None)
    args = ap.parse_args(argv)
    case = load_case(args.par, args.dem, args.cfl, args.max_dt)
    r = run_case(case, capacity=2_000_000)
    nr, nc = case.mesh.bed.shape
    print(f"{nr} x {nc} cells at {case.header.cellsize} m: {r['steps']} steps, "
          f"t = {r['t']:.1f} s, {r['wall_s']:.2f} s wall")
    print(f"  {'pt':>3}  {'x':>10}  {'y':>10}  {'peak_h':>10}  {'final_h':>10}")
    for p, (x, y) in enumerate(case.points):
        print(f"  {p + 1:>3}  {x:>10.1f}  {y:>10.1f}  {r['peaks'][p]:>10.4f}  "
              f"{r['finals'][p]:>10.4f}")
    comparisons = {}
    for path in args.reference_stage:
        ref = read_reference_stage(path)
        rows = []
        print(f"\nvs {os.path.basename(path)}")
        print(f"  {'pt':>3}  {'ref_peak':>10}  {'rmse':>10}  {'peak_bias':>10}  {'arrival_dt':>10}")
        for p in range(len(case.points)):
            c = compare_point(ref, p, r["times"], r["depths"][:, p], args.arrival_threshold)
            dt = (f"{c.sim_arrival - c.reference_arrival:+.1f} s"
                  if c.sim_arrival is not None and c.reference_arrival is not None else "never")
            print(f"  {p + 1:>3}  {c.reference_peak:>10.4f}  {c.rmse:>10.4f}  "
                  f"{c.peak_bias:>+10.4f}  {dt:>10}")
            rows.append(c.__dict__)
        comparisons[os.path.basename(path)] = rows
    if args.json:
        with open(args.json, "w") as f:
            json.dump(dict(cells=[nr, nc], steps=r["steps"], t=r["t"], wall_s=r["wall_s"],
                           rows_seen=r["rows_seen"], points=case.points,
                           peaks=r["peaks"].tolist(), finals=r["finals"].tolist(),
                           comparisons=comparisons), f, indent=1)
    return r


if __name__ == "__main__":
    main()
