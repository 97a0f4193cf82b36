"""Seeded synthetic workloads: determinism and the configured distributions."""
import numpy as np

from hydroflux_b200 import workloads
from hydroflux_b200.ensemble import ensemble_scenarios


def test_uniform_is_reproducible_and_in_range():
    a = workloads.uniform(7, 3, 1000, 2.0, 5.0)
    b = workloads.uniform(7, 3, 1000, 2.0, 5.0)
    assert np.array_equal(a, b) and a.min() >= 2.0 and a.max() < 5.0
    assert not np.array_equal(a, workloads.uniform(8, 3, 1000, 2.0, 5.0))
    assert abs(a.mean() - 3.5) < 0.1


def test_valley_generator():
    s = workloads.valley(n=256, dx=5.0, seed=1)
    assert s.shape == (256, 256) and np.all(s.h == 0.0)
    assert set(np.unique(s.manning)) <= set(workloads.MANNING_CLASSES)
    # without hills: 0.005 longitudinal descent to the south, 0.05 side slopes
    base = workloads.valley_bed(256, 5.0, 1, n_hills=0)
    assert abs((base[0, 128] - base[-1, 128]) - 0.005 * 255 * 5.0) < 1e-9
    # cell centres x = 2.5 m and 642.5 m, valley axis at 640 m
    assert abs((base[10, 0] - base[10, 128]) - 0.05 * (637.5 - 2.5)) < 1e-9
    assert s.sources[0][0] == 0 and s.sources[0][1] == 128
    t, q = s.sources[0][2], s.sources[0][3]
    assert q.max() == 500.0 and t[np.argmax(q)] == 1800.0
    assert abs(s.rain[1][0] - 50e-3 / 3600.0) < 1e-18
    assert np.array_equal(workloads.valley(n=64, seed=3).bed, workloads.valley(n=64, seed=3).bed)


def test_ensemble_scenarios_distribution():
    scns = ensemble_scenarios(count=64, seed=0, side_lo=16, side_hi=64, horizon=60.0)
    sides = np.array([s.shape[0] for s in scns])
    assert sides.min() >= 16 and sides.max() <= 64
    assert all(s.shape[0] == s.shape[1] for s in scns)
    ns = np.array([s.manning[0, 0] for s in scns])
    assert ns.min() >= 0.02 and ns.max() <= 0.08
    peaks = np.array([s.sources[0][3].max() for s in scns])
    assert peaks.min() >= 250.0 and peaks.max() <= 1000.0
    assert all(s.t_end == 60.0 for s in scns)
