"""max_depth_exceeds_relief (solver-2d/src/sim.rs:248-271) on the GPU: the
reference's two unit tests (sim.rs:376-397) through the simulation handle
and the free function, the fold semantics (NaN skipped, depth max from 0,
1 m relief floor) against the oracle on random fields, and a full-size
field whose decisive depth is the last cell."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hydroflux_b200 import sim, step
    return torch, sim, step


def _sim(sim, bed, h, dx=1.0, n=0.03):
    zero = np.zeros_like(h)
    return sim.Simulation(sim.Mesh2D(bed, dx, dx, n), (h, zero, zero), sim.SimulationConfig(),
                          device=0)


def test_flags_a_finite_blow_up(gpu):  # sim.rs:376-386
    torch, sim, step = gpu
    bed = np.repeat(np.arange(4, dtype=float)[:, None] * 32.0, 4, axis=1)  # 0..96 m
    with _sim(sim, bed, np.full((4, 4), 5.0), dx=30.0, n=0.035) as s:
        assert not s.max_depth_exceeds_relief(3.0)
    with _sim(sim, bed, np.full((4, 4), 3000.0), dx=30.0, n=0.035) as s:
        assert s.max_depth_exceeds_relief(3.0)


def test_floors_a_near_flat_mesh(gpu):  # sim.rs:388-397
    torch, sim, step = gpu
    bed = np.zeros((3, 3))
    with _sim(sim, bed, np.full((3, 3), 2.0)) as s:
        assert not s.max_depth_exceeds_relief(3.0)
    with _sim(sim, bed, np.full((3, 3), 50.0)) as s:
        assert s.max_depth_exceeds_relief(3.0)


@pytest.mark.parametrize("shape", [(1, 1), (5, 7), (64, 96), (257, 129)])
def test_free_function_matches_oracle(gpu, oracle, shape):
    """Random beds and depths with NaNs, negatives and infinities, factors
    around the decision point: the device reduction decides as the oracle."""
    torch, sim, step = gpu
    rng = np.random.default_rng(shape[0] * 1000 + shape[1])
    for trial in range(24):
        bed = rng.uniform(-50.0, 50.0, shape) * rng.choice([1e-3, 1.0, 10.0])
        h = rng.uniform(-1.0, 30.0, shape)
        if trial % 3 == 1:
            bed[rng.uniform(size=shape) < 0.2] = np.nan
            h[rng.uniform(size=shape) < 0.2] = np.nan
        if trial % 6 == 2:
            bed[:] = np.nan
        if trial % 8 == 5:
            h[:] = -1.0
        if trial == 7:
            bed.flat[-1] = np.inf
        relief = max(float(np.nanmax(bed)) - float(np.nanmin(bed)), 1.0) \
            if np.isfinite(bed).any() else 1.0
        hmax = max(float(np.nanmax(h)), 0.0) if not np.isnan(h).all() else 0.0
        for factor in (0.0, hmax / relief if np.isfinite(relief) and relief > 0 else 1.0,
                       np.nextafter(hmax / relief, np.inf) if np.isfinite(relief) else 2.0,
                       0.5, 3.0):
            mesh = step.DeviceMesh(bed, 1.0, 1.0, 0.03)
            got = step.max_depth_exceeds_relief(torch.tensor(h, device="cuda"), mesh, factor)
            want = oracle.max_depth_exceeds_relief(h, bed, factor)
            assert got == want, (shape, trial, factor)


def test_full_size_last_cell_decides(gpu, oracle):
    """2048 x 4096 cells: the one depth above the threshold is the last
    cell, so every block's partial must reach the result."""
    torch, sim, step = gpu
    nr, nc = 2048, 4096
    rng = np.random.default_rng(5)
    bed = rng.uniform(0.0, 10.0, (nr, nc))
    bed[0, 0], bed[-1, -1] = 0.0, 10.0
    h = rng.uniform(0.0, 20.0, (nr, nc))
    mesh = step.DeviceMesh(bed, 5.0, 5.0, 0.03)
    ht = torch.tensor(h, device="cuda")
    assert not step.max_depth_exceeds_relief(ht, mesh, 2.0)
    ht[-1, -1] = 20.5
    h[-1, -1] = 20.5
    assert step.max_depth_exceeds_relief(ht, mesh, 2.0)
    assert oracle.max_depth_exceeds_relief(h, bed, 2.0)
    with _sim(sim, bed, h, dx=5.0) as s:
        assert s.max_depth_exceeds_relief(2.0)
        assert not s.max_depth_exceeds_relief(2.05)
