"""LISFLOOD-FP deck readers and the run they build (host side, no GPU), and
the oracle's series units pinned to the reference examples' arithmetic."""
import math
import os

import numpy as np
import pytest

# The two UK EA decks are committed as fixtures (copied from the reference's
# benchmarks/data/uk_ea by tests/golden/make_golden.py).
UK_EA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "uk_ea")


@pytest.fixture(scope="module")
def L():
    from hydroflux_b200 import build
    build.build()
    from hydroflux_b200 import lisflood
    return lisflood


def write_deck(tmp_path, R, with_rain=True, bci_lines=("P 35.0 15.0 QVAR inflow",),
               manning_grid=True):
    hd = R.AsciiGridHeader(6, 4, 0.0, 0.0, 10.0, -9999.0)
    bed = np.arange(24, dtype=np.float64).reshape(4, 6) * 0.1
    R.write_ascii_grid(str(tmp_path / "d.dem.gz"), bed, hd)
    if manning_grid:
        R.write_ascii_grid(str(tmp_path / "d.n"), np.where(bed > 1.0, 0.05, 0.02), hd)
    par = ["DEMfile  d.dem", "bcifile d.bci", "bdyfile d.bdy", "stagefile d.stage",
           "sim_time 600.0", "acceleration", "# a comment line", "elevoff"]
    par.append("manningfile d.n" if manning_grid else "fpfric 0.03")
    if with_rain:
        par.append("rainfall d.rain")
        (tmp_path / "d.rain").write_text("# hyetograph\r\n3 minutes\r\n0 0\r\n100 1\r\n0 2\r\n")
    (tmp_path / "d.par").write_text("\n".join(par) + "\n")
    (tmp_path / "d.bci").write_text("\n".join(bci_lines) + "\n")
    (tmp_path / "d.bdy").write_text("# inflows\ninflow\n3 minutes\n0 0\n0.5 5\n0 10\n"
                                    "edge\n2 seconds\n0 0\n1 600\n")
    (tmp_path / "d.stage").write_text("2\n5 5\n55 35\n\n\n")
    return str(tmp_path / "d.par"), bed


def test_point_inflow_deck(L, tmp_path):
    from hydroflux_b200 import raster as R
    par, bed = write_deck(tmp_path, R)
    c = L.load_case(par, max_dt=10.0)
    assert c.mesh.bed.shape == (4, 6) and np.array_equal(c.mesh.bed, bed)
    assert sorted(np.unique(c.mesh.manning).tolist()) == [0.02, 0.05]
    assert c.sim_time == 600.0 and c.config.max_dt == 10.0 and c.config.cfl == 0.4
    assert all(b.kind == 1 for b in (c.config.boundaries.north, c.config.boundaries.south,
                                     c.config.boundaries.west, c.config.boundaries.east))
    assert len(c.sources) == 1
    r, col, t, v = c.sources[0]
    assert (r, col) == (2, 3)                 # cell_at(35, 15): row_from_south 1 -> row 2
    assert t.tolist() == [0.0, 5.0, 10.0] and v.tolist() == [0.0, 0.5, 0.0]
    assert c.source_units == (60.0, 10.0, 1.0)  # minutes; q = QVAR * cellsize
    assert c.rain[0].tolist() == [0.0, 1.0, 2.0] and c.rain[1].tolist() == [0.0, 100.0, 0.0]
    assert c.rain_units == (60.0, 1e-3, 3600.0)
    assert c.gauges == [(3, 0), (0, 5)]


def test_line_inflow_and_free_sides(L, tmp_path):
    from hydroflux_b200 import raster as R
    par, _ = write_deck(tmp_path, R, with_rain=False, manning_grid=False,
                        bci_lines=("W 12.0 31.0 QVAR edge", "E 0 40 FREE", "N 0 60 FREE"))
    c = L.load_case(par)
    b = c.config.boundaries
    assert (b.west.kind, b.east.kind, b.north.kind, b.south.kind) == (1, 0, 0, 1)
    assert np.all(c.mesh.manning == 0.03) and c.rain is None
    # rows overlapping y in [12, 31): south rows 1, 2, 3 -> rows 2, 1, 0, all at col 0
    assert [(s[0], s[1]) for s in c.sources] == [(2, 0), (1, 0), (0, 0)]
    assert c.source_units == (1.0, 19.0, 3.0)


def test_deck_errors(L, tmp_path):
    from hydroflux_b200 import raster as R
    par, _ = write_deck(tmp_path, R, bci_lines=("P 1000.0 15.0 QVAR inflow",))
    with pytest.raises(ValueError):
        L.load_case(par)
    par, _ = write_deck(tmp_path, R, bci_lines=("N 0 60 HFIX 1.0",))
    with pytest.raises(NotImplementedError):
        L.load_case(par)
    par, _ = write_deck(tmp_path, R, bci_lines=("P 35.0 15.0 QVAR inflow", "W 12 31 QVAR edge"))
    with pytest.raises(NotImplementedError):   # one units setting for all point sources
        L.load_case(par)


def test_interp_and_compare_point(L, tmp_path):
    assert L.interp([0.0, 10.0], [0.0, 1.0], -1.0) == 0.0
    assert L.interp([0.0, 10.0], [0.0, 1.0], 11.0) == 1.0
    assert L.interp([0.0, 10.0, 10.0, 20.0], [0.0, 1.0, 5.0, 5.0], 10.0) == 5.0  # last of equal stamps
    assert L.interp([0.0, 10.0], [2.0, 4.0], 2.5) == 2.5
    text = ("Stage output, depth (m). Stage locations from: x.stage\n\n"
            "Stage information (stage,x,y,elev):\n1\t5.0\t5.0\t0.0\n2\t55.0\t35.0\t0.0\n\n"
            "Output, depths:\nTime; stages 1 to 2\n   10.0  0.0  0.0\n   20.0  0.10  0.00\n"
            "   bad row here\n   30.0  0.30  0.03  9.9\n   40.0  0.20  0.05\n")
    p = tmp_path / "r.stage"
    p.write_text(text)
    ref = L.read_reference_stage(str(p))
    assert ref.points == [(5.0, 5.0), (55.0, 35.0)]
    assert ref.times.tolist() == [10.0, 20.0, 40.0]
    sim_t = [0.0, 15.0, 25.0, 45.0]
    sim_v = [0.0, 0.05, 0.15, 0.25]
    c = L.compare_point(ref, 0, sim_t, sim_v, 0.02)
    on_grid = [L.interp(sim_t, sim_v, t) for t in ref.times]
    want = math.sqrt(sum((r - s) ** 2 for r, s in zip([0.0, 0.1, 0.2], on_grid)) / 3)
    assert c.rmse == want and c.reference_peak == 0.2
    assert c.peak_bias == max(on_grid) - 0.2
    assert c.reference_arrival == 20.0 and c.sim_arrival == 10.0  # 0.033 > 0.02 at t = 10


def test_oracle_units_match_example_arithmetic(L, tmp_path, oracle):
    """The oracle's series units give, step by step, the rain and inflow the
    reference's urban example computes on the host:
    interp(t_s / 60) * 1e-3 / 3600 and interp(t_s / 60) * cellsize
    (solver-2d/examples/uk_ea_test8a_official.rs:119-134)."""
    from hydroflux_b200 import abi
    O = oracle
    rng = np.random.default_rng(5)
    nr, nc, dx = 12, 10, 2.0
    z = rng.uniform(0.0, 0.3, (nr, nc))
    n = np.full((nr, nc), 0.03)
    rain_t = np.array([0.0, 0.05, 0.1, 0.7, 0.9, 3.0])
    rain_v = np.array([0.0, 0.0, 400.0, 400.0, 37.0, 0.0])
    src_t = np.array([0.0, 0.2, 0.45, 1.1, 2.0])
    src_v = np.array([0.0, 0.03125, 0.65625, 2.3125, 0.0])
    cfg = abi.make_config(max_dt=2.0)
    f = O.Forcing(rain=(rain_t, rain_v), sources=[(4, 6, src_t, src_v)],
                  rain_units=(60.0, 1e-3, 3600.0), src_units=(60.0, dx, 1.0))
    zero = np.zeros((nr, nc))
    a = O.sim_run(z, n, dx, dx, zero, zero, zero, cfg, 150.0, forcing=f, stop_after=60,
                  dt_log_cap=60)
    assert a["status"] == 0 and a["steps"] == 60
    h, hu, hv, t = zero, zero, zero, 0.0
    for k in range(60):
        dt = a["dts"][k]
        t_new = t + dt
        rate = L.interp(rain_t, rain_v, t_new / 60.0) * 1e-3 / 3600.0
        q = L.interp(src_t, src_v, t_new / 60.0) * dx
        g = O.Forcing(rain=([0.0], [rate]), sources=[(4, 6, [0.0], [q])])
        s = O.sim_step(z, n, dx, dx, h, hu, hv, cfg, 150.0 - t, forcing=g, t0=t, steps0=k)
        assert s["status"] == 0 and s["dt"] == dt
        h, hu, hv, t = s["h"], s["hu"], s["hv"], s["t"]
    O.Forcing().args()  # restore the default units
    for x, y in ((a["h"], h), (a["hu"], hu), (a["hv"], hv)):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))
    assert a["t"] == t


@pytest.mark.parametrize("deck", ["test8a_glasgow/ea8-2m.par", "test4/ea4.par"])
def test_reference_decks(L, deck):
    path = os.path.join(UK_EA, deck)
    if deck.startswith("test8a"):
        c = L.load_case(path, max_dt=10.0)
        assert c.mesh.bed.shape == (199, 481) and len(c.gauges) == 9 and len(c.sources) == 1
        assert c.source_units == (60.0, 2.0, 1.0) and c.rain_units == (60.0, 1e-3, 3600.0)
        assert c.rain[1].max() == 400.0 and c.sources[0][3].max() == 2.5
    else:
        c = L.load_case(path, dem="ea4-5m.dem", max_dt=15.0)
        assert c.mesh.bed.shape == (400, 200) and np.all(c.mesh.bed == 0.0)
        assert np.all(c.mesh.manning == 0.05) and len(c.gauges) == 6
        assert [s[:2] for s in c.sources] == [(201, 0), (200, 0), (199, 0), (198, 0)]
        assert c.source_units == (1.0, 20.0, 4.0)
        b = c.config.boundaries
        assert (b.west.kind, b.east.kind, b.north.kind, b.south.kind) == (1, 0, 0, 0)
        for f in ("ea4-5m-dg2.stage", "ea4-1m-acc.stage"):
            ref = L.read_reference_stage(os.path.join(UK_EA, "test4/reference", f))
            assert ref.points == c.points and len(ref.times) > 100
    assert c.sim_time == 18000.0


def test_oracle_gauge_recorder(L, oracle):
    """The oracle's run records the same peaks and last depths as stepping
    it one step at a time (the check the GPU gauges are held to)."""
    from hydroflux_b200 import abi
    O = oracle
    rng = np.random.default_rng(13)
    nr, nc = 9, 11
    z = rng.uniform(0.0, 0.5, (nr, nc))
    n = np.full((nr, nc), 0.03)
    h0 = rng.uniform(0.0, 0.4, (nr, nc)) * (rng.uniform(size=(nr, nc)) > 0.3)
    zero = np.zeros((nr, nc))
    cfg = abi.make_config(max_dt=0.5)
    cells = [0, 5 * nc + 3, nr * nc - 1, 5 * nc + 3]
    r = O.sim_run(z, n, 1.0, 1.0, h0, zero, zero, cfg, 1e9, stop_after=40, gauges=cells)
    h, hu, hv, t = h0, zero, zero, 0.0
    peak = np.maximum(h0.ravel()[cells], 0.0)
    for k in range(40):
        s = O.sim_step(z, n, 1.0, 1.0, h, hu, hv, cfg, 1e9 - t, t0=t, steps0=k)
        h, hu, hv, t = s["h"], s["hu"], s["hv"], s["t"]
        peak = np.maximum(peak, h.ravel()[cells])
    assert np.array_equal(r["gauge_peak"], peak)
    assert np.array_equal(r["gauge_last"], h.ravel()[cells])
    assert np.array_equal(r["h"], h)
