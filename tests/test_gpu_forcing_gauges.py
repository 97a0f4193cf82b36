"""Forcing-series units and control-point gauges on the GPU, bitwise against
the oracle; and the LISFLOOD-FP benchmark decks on real terrain (the
committed tests/golden/uk_ea fixtures), GPU against the oracle over the
first steps of each event."""
import os

import numpy as np
import pytest

from tests.gpu_util import exact_fraction

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hydroflux_b200 import lisflood, sim
    return sim, lisflood


@pytest.fixture(autouse=True)
def libm_pow(oracle):
    oracle.set_pow_mode("libm")
    yield
    oracle.Forcing().args()  # default series units


def urban_like(nr=70, nc=90, seed=11):
    rng = np.random.default_rng(seed)
    z = 0.004 * np.arange(nr)[:, None] + 0.02 * np.abs(np.arange(nc) - nc / 3)[None, :] \
        + rng.uniform(0.0, 0.4, (nr, nc))
    n = np.where(rng.uniform(size=(nr, nc)) < 0.3, 0.02, 0.05)
    return z, n


RAIN = (np.array([0.0, 0.05, 0.1, 0.7, 0.9, 3.0]), np.array([0.0, 0.0, 400.0, 400.0, 37.0, 0.0]))
SRC = [(10, 20, np.array([0.0, 0.2, 0.45, 1.1, 2.0]), np.array([0.0, 0.03125, 0.65625, 2.3125, 0.0])),
       (50, 71, np.array([0.0, 0.3, 1.2]), np.array([0.0, 1.21875, 0.0])),
       (50, 71, np.array([0.0]), np.array([0.1]))]


def run_pair(sim, oracle, z, n, dx, cfg, n_steps, rain_units, src_units, gauges=None,
             capacity=1 << 16, src=SRC):
    zero = np.zeros_like(z)
    mesh = sim.Mesh2D(z, dx, dx, n)
    with sim.Simulation(mesh, (zero, zero, zero), cfg) as s:
        s.set_rain(np.stack(RAIN, axis=1))
        s.set_rain_units(*rain_units)
        s.set_point_sources([sim.PointSource(r, c, np.stack((t, v), axis=1)) for r, c, t, v in src])
        s.set_point_source_units(*src_units)
        if gauges is not None:
            s.set_gauges(gauges, capacity)
        s.run_steps(n_steps)
        got = s.states()
        out = dict(state=got, steps=s.steps(), t=s.time())
        if gauges is not None:
            out["peaks"], out["last"] = s.gauge_peaks()
            out["series"] = s.gauge_series()
    f = oracle.Forcing(rain=RAIN, sources=src, rain_units=rain_units, src_units=src_units)
    r = oracle.sim_run(z, n, dx, dx, zero, zero, zero, cfg.to_c(), 1e9, forcing=f,
                       stop_after=n_steps, dt_log_cap=n_steps)
    return out, r


@pytest.mark.parametrize("integrator", [0, 1])
def test_series_units_bitwise(gpu, oracle, integrator):
    """Rain in minutes and mm/h, (v * 1e-3) / 3600, and inflows in minutes
    times the cell size, evaluated on the device at t_new: bitwise equal to
    the oracle's host arithmetic."""
    sim, _ = gpu
    z, n = urban_like()
    cfg = sim.SimulationConfig(cfl=0.4, integrator=sim.Integrator(integrator), max_dt=2.0)
    out, r = run_pair(sim, oracle, z, n, 2.0, cfg, 400, (60.0, 1e-3, 3600.0), (60.0, 2.0, 1.0))
    assert r["status"] == 0 and out["steps"] == r["steps"] == 400 and out["t"] == r["t"]
    assert exact_fraction(out["state"], (r["h"], r["hu"], r["hv"])) == 1.0
    assert r["h"].max() > 0.01  # the forcing did something


def test_default_units_are_the_identity(gpu, oracle):
    sim, _ = gpu
    z, n = urban_like(60, 80, 3)
    cfg = sim.SimulationConfig(cfl=0.4, max_dt=2.0)
    out, r = run_pair(sim, oracle, z, n, 2.0, cfg, 150, (1.0, 1.0, 1.0), (1.0, 1.0, 1.0))
    assert exact_fraction(out["state"], (r["h"], r["hu"], r["hv"])) == 1.0
    # and the two-divisor form with a non-trivial divisor
    out, r = run_pair(sim, oracle, z, n, 2.0, cfg, 150, (7.0, 3.0, 11.0), (0.5, 1.7, 3.0))
    assert exact_fraction(out["state"], (r["h"], r["hu"], r["hv"])) == 1.0


def test_gauges_record_every_step(gpu, oracle):
    """Gauge rows are the depths after every step (row 0: the initial
    state), peaks are fold(0.0, f64::max) over all rows; rows beyond the
    capacity are counted, not stored."""
    sim, _ = gpu
    z, n = urban_like(30, 40, 7)
    dx = 2.0
    cfg = sim.SimulationConfig(cfl=0.4, max_dt=2.0)
    gauges = [(10, 20), (0, 0), (29, 39), (15, 7), (10, 20)]
    ru, su = (60.0, 1e-3, 3600.0), (60.0, dx, 1.0)
    n_steps, cap = 120, 50
    src = [SRC[0]]
    out, r = run_pair(sim, oracle, z, n, dx, cfg, n_steps, ru, su, gauges, cap, src)
    # oracle, one step at a time, sampling the gauges
    zero = np.zeros_like(z)
    h, hu, hv, t = zero, zero, zero, 0.0
    rows_t, rows_h = [0.0], [[0.0] * len(gauges)]
    f = oracle.Forcing(rain=RAIN, sources=src, rain_units=ru, src_units=su)
    for k in range(n_steps):
        s = oracle.sim_step(z, n, dx, dx, h, hu, hv, cfg.to_c(), 1e9 - t, forcing=f, t0=t,
                            steps0=k)
        assert s["status"] == 0
        h, hu, hv, t = s["h"], s["hu"], s["hv"], s["t"]
        rows_t.append(t)
        rows_h.append([h[g] for g in gauges])
    rows_t, rows_h = np.array(rows_t), np.array(rows_h)
    assert exact_fraction(out["state"], (r["h"], r["hu"], r["hv"])) == 1.0
    assert np.array_equal(out["state"][0], h)
    ts, hs, seen = out["series"]
    assert seen == n_steps + 1 and len(ts) == cap and hs.shape == (cap, len(gauges))
    assert np.array_equal(ts, rows_t[:cap]) and np.array_equal(hs, rows_h[:cap])
    assert np.array_equal(out["last"], rows_h[-1])
    assert np.array_equal(out["peaks"], np.maximum(rows_h.max(axis=0), 0.0))
    assert out["peaks"][0] > 0.0


def test_gauge_errors(gpu):
    sim, _ = gpu
    z = np.zeros((8, 9))
    with sim.Simulation(sim.Mesh2D(z, 1.0, 1.0, 0.03), (z + 0.1, z, z)) as s:
        with pytest.raises(ValueError):
            s.gauge_peaks()
        with pytest.raises(ValueError):
            s.set_gauges([(8, 0)])
        with pytest.raises(ValueError):
            s.set_gauges([(0, -1)])
        with pytest.raises(ValueError):
            s.set_rain_units(0.0, 1.0, 1.0)
        with pytest.raises(ValueError):
            s.set_point_source_units(1.0, 1.0, 0.0)
        s.set_gauges([(3, 4)], capacity=0)
        s.run_until(0.5)
        ts, hs, seen = s.gauge_series()
        assert len(ts) == 0 and seen == s.steps() + 1
        peaks, last = s.gauge_peaks()
        assert last[0] == s.states()[0][3, 4] and peaks[0] >= 0.1
        s.set_gauges([])
        with pytest.raises(ValueError):
            s.gauge_peaks()


# The decks are committed as fixtures (tests/golden/uk_ea, copied from the
# reference's benchmarks/data/uk_ea by tests/golden/make_golden.py);
# HYDROFLUX_UK_EA_DIR may name another copy.
UK_EA = os.environ.get("HYDROFLUX_UK_EA_DIR") or os.path.join(
    os.path.dirname(os.path.abspath(__file__)), "golden", "uk_ea")
DECKS = [("test8a_glasgow/ea8-2m.par", None, 10.0, 1500),
         ("test4/ea4.par", "ea4-5m.dem", 15.0, 1500)]


@pytest.mark.parametrize("deck,dem,max_dt,n_steps", DECKS)
def test_real_terrain_decks(gpu, oracle, deck, dem, max_dt, n_steps):
    """The UK EA decks (urban rain + point inflow on a 481 x 199 DEM; line
    inflow over a 400 x 200 floodplain), first steps of each event, GPU
    against the oracle bitwise, gauges included."""
    assert os.path.exists(os.path.join(UK_EA, deck)), f"deck fixture missing under {UK_EA}"
    sim, L = gpu
    case = L.load_case(os.path.join(UK_EA, deck), dem=dem, max_dt=max_dt)
    s = L.simulation(case)
    s.run_steps(n_steps)
    got = s.states()
    peaks, last = s.gauge_peaks()
    ts, hs, seen = s.gauge_series()
    t_gpu, steps = s.time(), s.steps()
    s.close()
    zero = np.zeros_like(case.mesh.bed)
    f = oracle.Forcing(rain=case.rain, sources=case.sources, rain_units=case.rain_units,
                       src_units=case.source_units)
    r = oracle.sim_run(case.mesh.bed, case.mesh.manning, case.mesh.dx, case.mesh.dy, zero, zero,
                       zero, case.config.to_c(), case.sim_time, forcing=f, stop_after=n_steps)
    assert r["status"] == 0 and steps == r["steps"] == n_steps and t_gpu == r["t"]
    assert exact_fraction(got, (r["h"], r["hu"], r["hv"])) == 1.0
    assert seen == n_steps + 1 and ts[-1] == t_gpu
    assert np.array_equal(last, [r["h"][g] for g in case.gauges])
    assert np.array_equal(peaks, np.maximum(hs.max(axis=0), 0.0))
    assert r["h"].sum() > 0.0
