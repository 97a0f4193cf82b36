"""The streaming strip stage kernel (hf_strip.cuh, HF_STAGE_STRIP) against the
tile kernel (HF_STAGE_TILE) and the oracle.

The strip kernel carries halo rows from one 7-row block to the next down a
32-column strip, fetches new rows with TMA, and starts from scratch where a
CTA's range of blocks begins or enters a new strip. It must give the tile
kernel's results bit for bit: shapes below, at and above the block height,
strip widths with and without a partial last strip, interior and edge
blocks, every boundary kind, rain and point sources (repeated in one cell,
in several blocks), both integrators.
"""
import numpy as np
import pytest

from tests.gpu_util import assert_parity, exact_fraction
from tests.test_gpu_parity import BC_SETS, bcs_valid, random_case

pytestmark = pytest.mark.gpu

# rows: < 7, 7, 8, 14, 15, long; columns: even only (TMA rows start on 16
# bytes), one strip, one strip + a partial one, several strips
SHAPES = [(2, 2), (6, 32), (7, 32), (8, 34), (14, 64), (15, 66), (33, 96), (50, 130),
          (101, 70), (300, 40), (64, 256), (129, 200)]


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hydroflux_b200 import sim
    return sim


def run(sim, kind, z, n, state, cfg, steps, rain=None, sources=None):
    with sim.Simulation(sim.Mesh2D(z, 2.0, 1.5, n), state, cfg) as s:
        s.set_stage_kernel(kind)
        assert s.stage_kernel() == kind
        if rain is not None:
            s.set_rain(rain)
        if sources:
            s.set_point_sources(sources)
        s.run_steps(steps)
        return s.states(), s.steps(), s.time()


@pytest.mark.parametrize("bc", sorted(BC_SETS))
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}")
def test_strip_equals_tile(gpu, shape, bc):
    sim = gpu
    nr, nc = shape
    pairs = BC_SETS[bc]
    if not bcs_valid(pairs, nr, nc):
        pytest.skip("Discharge/Depth need two cells normal to the side")
    z, n, h, hu, hv = random_case(nr, nc, seed=nr * 1000 + nc + len(bc))
    cfg = sim.SimulationConfig(cfl=0.45, max_dt=0.5, boundaries=sim.Boundaries2D(
        *[sim.Boundary(k, v) for k, v in pairs]))
    a = run(sim, "tile", z, n, (h, hu, hv), cfg, 12)
    b = run(sim, "strip", z, n, (h, hu, hv), cfg, 12)
    assert a[1] == b[1] == 12 and a[2] == b[2]
    assert exact_fraction(b[0], a[0]) == 1.0


@pytest.mark.parametrize("integrator", [0, 1])
def test_strip_forcing_against_oracle(gpu, oracle, integrator):
    """Rain and point sources (two in one cell, others in different blocks
    and strips, one on a block's first and one on its last row) on a dry
    valley, strip kernel against the oracle and the tile kernel, bitwise."""
    sim = gpu
    nr, nc = 71, 98
    rng = np.random.default_rng(7 + integrator)
    z = 0.01 * np.arange(nr)[:, None] + 0.05 * np.abs(np.arange(nc) - nc / 2)[None, :] \
        + rng.uniform(0, 0.05, (nr, nc))
    n = rng.choice([0.025, 0.035, 0.05, 0.08], size=(nr, nc))
    zeros = np.zeros((nr, nc))
    rain = ((0.0, 0.0), (5.0, 1e-3), (20.0, 1e-3), (20.0, 0.0))
    series = ((0.0, 0.0), (10.0, 4.0), (30.0, 0.0))
    cells = [(2, nc // 2), (2, nc // 2), (7, 31), (13, 32), (70, 97), (35, 64), (0, 0)]
    sources = [sim.PointSource(r, c, series if k % 2 == 0 else 0.5)
               for k, (r, c) in enumerate(cells)]
    bcs = sim.Boundaries2D(sim.Boundary.wall(), sim.Boundary.transmissive(),
                           sim.Boundary.transmissive(), sim.Boundary.wall())
    cfg = sim.SimulationConfig(cfl=0.5, integrator=sim.Integrator(integrator), boundaries=bcs,
                               max_dt=2.0)
    got = run(sim, "strip", z, n, (zeros, zeros, zeros), cfg, 60, rain=rain, sources=sources)
    tile = run(sim, "tile", z, n, (zeros, zeros, zeros), cfg, 60, rain=rain, sources=sources)
    assert exact_fraction(got[0], tile[0]) == 1.0
    from oracle.oracle import Forcing
    st, sq = np.array([p[0] for p in series]), np.array([p[1] for p in series])
    f = Forcing(rain=(np.array([p[0] for p in rain]), np.array([p[1] for p in rain])),
                sources=[(r, c, st, sq) if k % 2 == 0 else (r, c, np.array([0.0]), np.array([0.5]))
                         for k, (r, c) in enumerate(cells)])
    r = oracle.sim_run(z, n, 2.0, 1.5, zeros, zeros, zeros, cfg.to_c(), float("inf"), forcing=f,
                       stop_after=60)
    assert r["status"] == 0 and r["steps"] == got[1] == 60 and r["t"] == got[2]
    assert_parity(got[0], (r["h"], r["hu"], r["hv"]))
    assert exact_fraction(got[0], (r["h"], r["hu"], r["hv"])) == 1.0


def test_strip_selection(gpu):
    """The default is a tile kernel (32 x 32 tiles on a large grid, 32 x 8 on
    a small one); the strip kernel is taken when asked for, on any grid with
    an even column count."""
    sim = gpu
    zero = np.zeros((2048, 2048))
    with sim.Simulation(sim.Mesh2D(zero, 1.0, 1.0, 0.03), (zero + 1.0, zero, zero),
                        sim.SimulationConfig()) as s:
        assert s.stage_kernel() == "tile32"
        s.set_stage_kernel("strip")
        assert s.stage_kernel() == "strip"
        s.set_stage_kernel("auto")
        assert s.stage_kernel() == "tile32"
    small = np.zeros((64, 64))
    with sim.Simulation(sim.Mesh2D(small, 1.0, 1.0, 0.03), (small + 1.0, small, small),
                        sim.SimulationConfig()) as s:
        assert s.stage_kernel() == "tile"
        s.set_stage_kernel("strip")
        assert s.stage_kernel() == "strip"
        s.set_stage_kernel("auto")
        assert s.stage_kernel() == "tile"
    odd = np.zeros((64, 65))
    with sim.Simulation(sim.Mesh2D(odd, 1.0, 1.0, 0.03), (odd + 1.0, odd, odd),
                        sim.SimulationConfig()) as s:
        with pytest.raises(sim.SimError):
            s.set_stage_kernel("strip")
        assert s.stage_kernel() == "tile"
        s.run_steps(3)


@pytest.mark.parametrize("case", ["mostly_dry", "dry_start"])
def test_strip_dry_blocks_and_dynamic_schedule(gpu, case):
    """Dry interior blocks write their zero slopes and faces instead of
    computing them; once a step has skipped many of them, the next steps
    claim blocks dynamically. The mostly-dry channel valley of the reference's
    criterion bench (6% wet) and the valley flood from its dry start (rain
    and inflow wet the blocks step by step) give the tile kernel's results
    bit for bit."""
    sim = gpu
    from hydroflux_b200 import workloads
    if case == "mostly_dry":
        s = workloads.step_regime("mostly_dry", 512)
        steps = 15
    else:
        s = workloads.valley(n=384, dx=5.0, seed=2, t_end=1e9)
        steps = 25
    out = {}
    for kind in ("tile", "strip"):
        with workloads.simulation_for(s) as sm:
            sm.set_stage_kernel(kind)
            sm.run_steps(steps, s.t_end)
            out[kind] = (sm.states(), sm.steps(), sm.time())
    assert out["tile"][1] == out["strip"][1] == steps and out["tile"][2] == out["strip"][2]
    assert exact_fraction(out["strip"][0], out["tile"][0]) == 1.0
