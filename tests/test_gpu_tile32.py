"""The 32 x 32 tile geometry of the stage kernels (HF_STAGE_TILE32: 1024
threads, one CTA per SM) against the 32 x 8 one (HF_STAGE_TILE) and the
oracle.

Both geometries run the same phases on every cell; only the tiles, the
halo recomputation and the point-source buckets differ. Results must be
identical bit for bit: shapes below, at and above one tile, partial last
tiles in both directions, interior and edge tiles, every boundary kind,
rain and point sources (repeated in one cell, on tile edges), both
integrators. Grids of at least 100 such tiles take this geometry by default,
and so do ensembles whose scenarios add up to that many and every server.
"""
import numpy as np
import pytest

from tests.gpu_util import assert_parity, exact_fraction
from tests.test_gpu_parity import BC_SETS, bcs_valid, random_case

pytestmark = pytest.mark.gpu

# one tile and less, one tile plus one cell, the interior-tile threshold (the
# tile at (32, 32) has its 4-cell halo inside a grid of 68 x 68; 67 rows
# leave it on the edge path), interior tiles with partial last tiles, thin
# grids
SHAPES = [(1, 1), (3, 5), (31, 32), (32, 32), (33, 33), (40, 41), (67, 68), (68, 68),
          (72, 64), (97, 130), (130, 70), (200, 33), (5, 300), (300, 5)]


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


@pytest.mark.parametrize("integrator", [0, 1])
@pytest.mark.parametrize("bc", sorted(BC_SETS))
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}")
def test_tile32_equals_tile(gpu, shape, bc, integrator):
    sim = gpu
    nr, nc = shape
    pairs = BC_SETS[bc]
    if not bcs_valid(pairs, nr, nc):
        pytest.skip("Discharge/Depth need two cells normal to the side")
    z, n, h, hu, hv = random_case(nr, nc, seed=nr * 1000 + nc + len(bc))
    cfg = sim.SimulationConfig(cfl=0.45, max_dt=0.5, integrator=sim.Integrator(integrator),
                               boundaries=sim.Boundaries2D(
                                   *[sim.Boundary(k, v) for k, v in pairs]))
    a = run(sim, "tile", z, n, (h, hu, hv), cfg, 10)
    b = run(sim, "tile32", z, n, (h, hu, hv), cfg, 10)
    assert a[1] == b[1] == 10 and a[2] == b[2]
    assert exact_fraction(b[0], a[0]) == 1.0


@pytest.mark.parametrize("integrator", [0, 1])
def test_tile32_forcing_against_oracle(gpu, oracle, integrator):
    """Rain and point sources (two in one cell, others on the first and last
    rows and columns of 32 x 32 tiles and in a partial tile) on a dry valley,
    32 x 32 tiles against the oracle and the 32 x 8 tiles, bitwise."""
    sim = gpu
    nr, nc = 75, 98
    rng = np.random.default_rng(11 + integrator)
    z = 0.01 * np.arange(nr)[:, None] + 0.05 * np.abs(np.arange(nc) - nc / 2)[None, :] \
        + rng.uniform(0, 0.05, (nr, nc))
    n = rng.choice([0.025, 0.035, 0.05, 0.08], size=(nr, nc))
    zeros = np.zeros((nr, nc))
    rain = ((0.0, 0.0), (5.0, 1e-3), (20.0, 1e-3), (20.0, 0.0))
    series = ((0.0, 0.0), (10.0, 4.0), (30.0, 0.0))
    cells = [(2, nc // 2), (2, nc // 2), (31, 31), (32, 32), (63, 64), (74, 97), (40, 96),
             (0, 0)]
    sources = [sim.PointSource(r, c, series if k % 2 == 0 else 0.5)
               for k, (r, c) in enumerate(cells)]
    bcs = sim.Boundaries2D(sim.Boundary.wall(), sim.Boundary.transmissive(),
                           sim.Boundary.transmissive(), sim.Boundary.wall())
    cfg = sim.SimulationConfig(cfl=0.5, integrator=sim.Integrator(integrator), boundaries=bcs,
                               max_dt=2.0)
    got = run(sim, "tile32", z, n, (zeros, zeros, zeros), cfg, 60, rain=rain, sources=sources)
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


def test_geometry_choice(gpu):
    """auto takes 32 x 32 tiles from 100 of them on (320 x 320 and 1 x 3169
    have exactly 100, partial tiles included), 32 x 8 below; either can be
    forced on any grid."""
    sim = gpu
    for shape, expect in (((320, 320), "tile32"), ((288, 320), "tile"), ((64, 64), "tile"),
                          ((2048, 2048), "tile32"), ((32, 3200), "tile32"), ((31, 3200), "tile32"),
                          ((1, 3168), "tile"), ((1, 3169), "tile32")):
        zero = np.zeros(shape)
        with sim.Simulation(sim.Mesh2D(zero, 1.0, 1.0, 0.03), (zero + 1.0, zero, zero),
                            sim.SimulationConfig()) as s:
            assert s.stage_kernel() == expect, shape
            other = "tile" if expect == "tile32" else "tile32"
            s.set_stage_kernel(other)
            assert s.stage_kernel() == other
            s.run_steps(2)
            s.set_stage_kernel("auto")
            assert s.stage_kernel() == expect


def test_full_size_valley_geometries_agree(gpu):
    """The 1024 x 1024 valley flood from its dry start (rain and inflow wet
    the tiles step by step; dry 32 x 32 tiles skip their faces) gives the same
    bits on both geometries."""
    sim = gpu
    from hydroflux_b200 import workloads
    s = workloads.valley(n=1024, dx=5.0, seed=5, t_end=1e9)
    out = {}
    for kind in ("tile", "tile32"):
        with workloads.simulation_for(s) as sm:
            sm.set_stage_kernel(kind)
            sm.run_steps(40, s.t_end)
            out[kind] = (sm.states(), sm.steps(), sm.time())
    assert out["tile"][1] == out["tile32"][1] == 40 and out["tile"][2] == out["tile32"][2]
    assert exact_fraction(out["tile32"][0], out["tile"][0]) == 1.0
