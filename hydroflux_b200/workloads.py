"""Seeded synthetic workloads (no datasets: every input is generated).

* `dam_break(n)` -- circular dam break: n x n, dx = 1 m, flat bed, h = 10 m
  within 50 m of the centre and 1 m outside, n = 0.03, walls, CFL 0.5.
* `valley(n, dx, seed)` -- flood in a synthetic valley: longitudinal slope
  0.005 descending toward the south (outflow) side, side slopes
  0.05 |x - x_c|, 200 Gaussian hills (height U[1, 20] m, sigma U[20, 200] m,
  uniform centres), Manning n from 4 Voronoi land-cover patches over
  {0.025, 0.035, 0.05, 0.08}, initially dry, one point inflow at the
  upstream thalweg with a triangular hydrograph 0 -> peak at 30 min -> 0 at
  60 min, rain 50 mm/h everywhere, transmissive (open) sides, CFL 0.5.
* `calibration_problem(n)` -- the valley with a smooth log-normal Manning
  field (median 0.04, sigma 0.3, 10-cell correlation), 16 thalweg gauges and
  a hidden Manning field of the same law that makes the observations.

Random numbers come from splitmix64 keyed by (seed, stream, index), so
every generator is reproducible element by element.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

RAIN_50MM_H = 50.0e-3 / 3600.0
MANNING_CLASSES = (0.025, 0.035, 0.05, 0.08)

_M64 = (1 << 64) - 1


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finalizer on uint64 arrays (wrapping arithmetic)."""
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, stream: int, count: int, lo=0.0, hi=1.0) -> np.ndarray:
    """`count` uniforms in [lo, hi) from (seed, stream)."""
    key = (int(seed) * 0x100000001B3 + int(stream) * 0x9E3779B1) & _M64
    idx = np.arange(count, dtype=np.uint64) + np.uint64(key)
    bits = splitmix64(idx) >> np.uint64(11)
    u = bits.astype(np.float64) * (1.0 / (1 << 53))
    return lo + (hi - lo) * u


@dataclass
class Scenario:
    """Mesh, initial state, boundaries and forcings of one solve."""
    name: str
    bed: np.ndarray
    manning: np.ndarray
    dx: float
    dy: float
    h: np.ndarray
    hu: np.ndarray
    hv: np.ndarray
    bcs: Tuple = ((1, 0.0),) * 4  # (kind, value) north, south, west, east
    cfl: float = 0.4
    t_end: float = 0.0
    max_dt: float = 60.0
    rain: Optional[Tuple[np.ndarray, np.ndarray]] = None          # (t, rate)
    integrator: int = 1  # 0 forward Euler, 1 SSP-RK2
    sources: List[Tuple[int, int, np.ndarray, np.ndarray]] = field(default_factory=list)

    @property
    def shape(self):
        return self.bed.shape

    @property
    def n_cells(self):
        return int(self.bed.size)


def dam_break(n: int = 256) -> Scenario:
    xc = np.arange(n) + 0.5
    X, Y = np.meshgrid(xc, xc)
    r = np.sqrt((X - n / 2.0) ** 2 + (Y - n / 2.0) ** 2)
    h = np.where(r < 50.0, 10.0, 1.0)
    z = np.zeros((n, n))
    return Scenario("dam_break", z, np.full_like(z, 0.03), 1.0, 1.0, h, np.zeros_like(h),
                    np.zeros_like(h), bcs=((1, 0.0),) * 4, cfl=0.5, t_end=10.0)


def valley_bed(n: int, dx: float, seed: int, n_hills: int = 200) -> np.ndarray:
    L = n * dx
    y = (np.arange(n) + 0.5) * dx  # along i (south = downstream)
    x = (np.arange(n) + 0.5) * dx
    bed = (0.005 * (L - y))[:, None] + (0.05 * np.abs(x - L / 2.0))[None, :]
    amp = uniform(seed, 1, n_hills, 1.0, 20.0)
    sig = uniform(seed, 2, n_hills, 20.0, 200.0)
    cx = uniform(seed, 3, n_hills, 0.0, L)
    cy = uniform(seed, 4, n_hills, 0.0, L)
    for a, s, hx, hy in zip(amp, sig, cx, cy):
        # Window of +-6 sigma (the Gaussian is below 1.6e-8 of its peak beyond).
        r = 6.0 * s
        j0, j1 = max(int((hx - r) / dx), 0), min(int((hx + r) / dx) + 1, n)
        i0, i1 = max(int((hy - r) / dx), 0), min(int((hy + r) / dx) + 1, n)
        if j0 >= j1 or i0 >= i1:
            continue
        gx = np.exp(-((x[j0:j1] - hx) ** 2) / (2.0 * s * s))
        gy = np.exp(-((y[i0:i1] - hy) ** 2) / (2.0 * s * s))
        bed[i0:i1, j0:j1] += a * np.outer(gy, gx)
    return bed


def voronoi_manning(n: int, dx: float, seed: int, classes=MANNING_CLASSES) -> np.ndarray:
    L = n * dx
    k = len(classes)
    sx = uniform(seed, 5, k, 0.0, L)
    sy = uniform(seed, 6, k, 0.0, L)
    x = (np.arange(n) + 0.5) * dx
    y = (np.arange(n) + 0.5) * dx
    best = np.full((n, n), np.inf)
    out = np.empty((n, n))
    for c in range(k):
        d = (y[:, None] - sy[c]) ** 2 + (x[None, :] - sx[c]) ** 2
        m = d < best
        best[m] = d[m]
        out[m] = classes[c]
    return out


def triangular_hydrograph(peak: float, t_peak: float = 1800.0, t_end: float = 3600.0):
    return np.array([0.0, t_peak, t_end]), np.array([0.0, peak, 0.0])


def valley(n: int = 4096, dx: float = 5.0, seed: int = 0, peak: float = 500.0,
           t_end: float = 3600.0, manning: Optional[np.ndarray] = None,
           rain_rate: float = RAIN_50MM_H) -> Scenario:
    bed = valley_bed(n, dx, seed)
    man = voronoi_manning(n, dx, seed) if manning is None else manning
    z0 = np.zeros((n, n))
    t, q = triangular_hydrograph(peak)
    sources = [(0, n // 2, t, q)]
    rain = (np.array([0.0]), np.array([rain_rate]))
    return Scenario(f"valley{n}", bed, man, dx, dx, z0, z0.copy(), z0.copy(),
                    bcs=((0, 0.0),) * 4, cfl=0.5, t_end=t_end, rain=rain, sources=sources)


def gaussian_smooth(a: np.ndarray, sigma: float) -> np.ndarray:
    """Separable Gaussian filter (kernel truncated at 4 sigma, edges reflected)."""
    r = int(np.ceil(4.0 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-x * x / (2.0 * sigma * sigma))
    k /= k.sum()
    out = a
    for axis in (0, 1):
        p = np.pad(out, [(r, r) if ax == axis else (0, 0) for ax in (0, 1)], mode="reflect")
        acc = np.zeros_like(out)
        n = out.shape[axis]
        for i, w in enumerate(k):
            acc += w * (p[i:i + n, :] if axis == 0 else p[:, i:i + n])
        out = acc
    return out


def lognormal_manning(n: int, seed: int, median: float = 0.04, sigma: float = 0.3,
                      corr_cells: float = 10.0) -> np.ndarray:
    """Per-cell Manning field with log n = ln(median) + sigma * g, g a smooth
    Gaussian field: white noise (Box-Muller on the seeded uniforms) filtered by
    a Gaussian of `corr_cells` cells and rescaled to unit variance."""
    u1 = uniform(seed, 7, n * n)
    u2 = uniform(seed, 8, n * n)
    w = (np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)).reshape(n, n)
    g = gaussian_smooth(w, corr_cells)
    g = (g - g.mean()) / g.std()
    return np.exp(np.log(median) + sigma * g)


@dataclass
class CalibrationProblem:
    """Gauge-misfit calibration of the Manning field on a valley flood."""
    scenario: Scenario        # its manning is the starting field
    n_steps: int
    gauges: np.ndarray        # row-major cell indices
    manning_true: np.ndarray  # hidden field that makes the observations


def calibration_problem(n: int = 512, dx: float = 5.0, seed: int = 0, n_steps: int = 2000,
                        n_gauges: int = 16, hidden_seed: Optional[int] = None,
                        t_end: float = 1.0e9) -> CalibrationProblem:
    """The valley flood (bed, inflow, rain, open sides as `valley`) with a
    log-normal Manning field (median 0.04, sigma 0.3, smoothed over 10 cells)
    to calibrate against gauge depths made with a hidden field of the same
    law. Gauges: `n_gauges` seeded rows of the valley's middle three
    quarters, each at the lowest bed cell within n/16 of the thalweg column
    (n/2), which the inflow and rain wet first. The run is `n_steps` steps
    (t_end far away)."""
    s = valley(n, dx, seed, t_end=t_end)
    s.manning = lognormal_manning(n, seed)
    hidden = lognormal_manning(n, seed + 1000 if hidden_seed is None else hidden_seed)
    rows = np.unique((uniform(seed, 9, 4 * n_gauges) * (0.75 * n)).astype(int) + n // 8)
    rows = np.sort(rows[:n_gauges])
    w = max(n // 16, 1)
    c0 = n // 2
    cols = [c0 - w + int(np.argmin(s.bed[r, c0 - w:c0 + w + 1])) for r in rows]
    gauges = np.array([r * n + c for r, c in zip(rows, cols)], dtype=np.int64)
    return CalibrationProblem(s, int(n_steps), gauges, hidden)


def step_regime(kind: str, n: int = 4096) -> Scenario:
    """The reference's two criterion regimes of the step
    (solver-2d/benches/step.rs:44-75), on an n x n grid of 1 m cells, Manning
    0.03, walls, CFL 0.4, no forcing. The reference runs them at 256 x 256;
    here the mostly-dry valley keeps its wet fraction at any n (the water
    level scales with n / 256, so the wet channel stays 1/16 of the width).

    all_wet: flat bed, h = 1 + 0.2 i/n + 0.1 j/n, hu = 0.1 h, hv = 0.05 h.
    mostly_dry: bed 0.05 |j - n/2|, level 0.4 n/256, h = max(level - z, 0),
    hu = 0, hv = 0.1 h (6.25% of the cells wet, in one channel strip)."""
    i = np.arange(n, dtype=np.float64)[:, None]
    j = np.arange(n, dtype=np.float64)[None, :]
    if kind == "all_wet":
        bed = np.zeros((n, n))
        h = 1.0 + 0.2 * (i / n) + 0.1 * (j / n)
        hu, hv = 0.1 * h, 0.05 * h
    elif kind == "mostly_dry":
        bed = np.broadcast_to(0.05 * np.abs(j - n / 2.0), (n, n)).copy()
        h = np.maximum(0.4 * n / 256.0 - bed, 0.0)
        hu, hv = np.zeros((n, n)), 0.1 * h
    else:
        raise ValueError(f"unknown regime {kind!r}")
    return Scenario(kind, bed, np.full((n, n), 0.03), 1.0, 1.0, h, hu, hv,
                    bcs=((1, 0.0),) * 4, cfl=0.4, t_end=float("inf"), max_dt=60.0)


def simulation_for(s: Scenario, device: int = 0, integrator=None):
    """A hydroflux_b200.sim.Simulation set up with the scenario's forcings."""
    from . import sim as S
    cfg = S.SimulationConfig(cfl=s.cfl, boundaries=S.Boundaries2D(*[S.Boundary(k, v)
                                                                    for k, v in s.bcs]),
                             max_dt=s.max_dt)
    if integrator is not None:
        cfg.integrator = integrator
    sm = S.Simulation(S.Mesh2D(s.bed, s.dx, s.dy, s.manning), (s.h, s.hu, s.hv), cfg, device)
    if s.rain is not None:
        sm.set_rain(np.stack(s.rain, axis=1))
    if s.sources:
        sm.set_point_sources([S.PointSource(r, c, np.stack([t, q], axis=1))
                              for r, c, t, q in s.sources])
    return sm


def oracle_forcing(s: Scenario):
    """The same forcings as the oracle's Forcing descriptor (test/bench use)."""
    from oracle.oracle import Forcing
    return Forcing(rain=s.rain, sources=s.sources)
