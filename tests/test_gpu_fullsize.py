"""The benchmark's 4096 x 4096 valley at full size.

* Twelve SSP-RK2 steps (rain, point inflow, Manning friction, transmissive
  sides) from the dry start, through the wetting of every cell: the GPU
  against the oracle (host libm pow) bit for bit, 16.8 M cells, the same dt
  sequence.
* The batched stage (an ensemble of this one scenario) against the
  single-grid stage on the same input, bit for bit: two different kernels
  and tile schedules over every interior and edge tile of the grid.
* Properties that need no oracle, at the same size: still water over the
  valley's bed stays still (the well-balanced property), and walls keep the
  mass.
"""
import dataclasses
import os

import numpy as np
import pytest

from tests.gpu_util import exact_fraction

pytestmark = pytest.mark.gpu

N = 4096


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hydroflux_b200 import ensemble, sim, workloads
    return sim, workloads, ensemble


@pytest.fixture(scope="module")
def warmed(gpu):
    """The benchmark's workload after 8 steps from its dry start (the
    inflow and the rain have wetted every cell), as a scenario that starts
    from that state at t = 0."""
    _, workloads, _ = gpu
    scn = workloads.valley(n=N, dx=5.0, seed=0)
    with workloads.simulation_for(scn) as s:
        s.run_steps(8, scn.t_end)
        h, hu, hv = s.states()
    return dataclasses.replace(scn, h=h, hu=hu, hv=hv)


def test_dry_start_bitwise_against_oracle(gpu, oracle):
    """The workload from its dry start at t = 0: rain (50 mm/h) and the
    inflow hydrograph wet the dry valley, so the first steps cross the dry
    and velocity thresholds in every cell. After 1, 4 and 12 steps the GPU
    equals the oracle (the host libm's pow, the reference's arithmetic) bit
    for bit, with the same clock."""
    _, workloads, ensemble = gpu
    scn = workloads.valley(n=N, dx=5.0, seed=0)
    assert float(np.max(scn.h)) == 0.0  # dry start
    cfg = ensemble.scenario_config(scn)
    forcing = workloads.oracle_forcing(scn)
    threads = oracle.get_threads()
    oracle.set_pow_mode("libm")
    oracle.set_threads(os.cpu_count() or 1)
    try:
        state, t0, k0 = (scn.h, scn.hu, scn.hv), 0.0, 0
        with workloads.simulation_for(scn) as sm:
            for k in (1, 4, 12):
                sm.run_steps(k - sm.steps(), scn.t_end)
                got = sm.states()
                r = oracle.sim_run(scn.bed, scn.manning, scn.dx, scn.dy, *state, cfg, scn.t_end,
                                   forcing=forcing, stop_after=k - k0, t0=t0, steps0=k0)
                assert r["status"] == 0 and r["steps"] == sm.steps() == k
                assert r["t"] == sm.time()
                assert exact_fraction(got, (r["h"], r["hu"], r["hv"])) == 1.0, f"after {k} steps"
                state, t0, k0 = (r["h"], r["hu"], r["hv"]), r["t"], r["steps"]
        assert float((state[0] > 1e-6).mean()) > 0.99  # every cell wetted
    finally:
        oracle.set_threads(threads)


def test_batched_stage_matches_single_grid_stage(gpu, warmed):
    _, workloads, ensemble = gpu
    s = warmed
    with workloads.simulation_for(s) as sm:
        sm.run_steps(3, s.t_end)
        ref, t = sm.states(), sm.time()
    with ensemble.Ensemble([s]) as ens:
        ens.run(3)
        info = ens.info(0)
        got = ens.states(0)
    assert info["steps"] == 3 and info["t"] == t
    assert exact_fraction(got, ref) == 1.0


def test_lake_at_rest_full_size(gpu, warmed):
    """Still water over the valley's relief scaled to 0.6 m (depths 0.2 to
    0.8 m, the scale at which the well-balanced test of the small grids
    holds its 1e-13), walls, no forcing: after 20 steps the surface is flat
    and the momentum zero to 1e-13, and the mass is kept to 1e-12."""
    sim, _, _ = gpu
    z = warmed.bed
    z = (z - z.min()) * (0.6 / (z.max() - z.min()))
    eta = float(z.max()) + 0.2
    h = eta - z
    zero = np.zeros_like(h)
    cfg = sim.SimulationConfig(cfl=0.45, max_dt=5.0)
    with sim.Simulation(sim.Mesh2D(z, 5.0, 5.0, warmed.manning), (h, zero, zero), cfg) as s:
        s.run_steps(20)
        got = s.states()
        assert s.steps() == 20
    assert np.max(np.abs(got[1])) <= 1e-13 and np.max(np.abs(got[2])) <= 1e-13
    assert np.max(np.abs(got[0] + z - eta)) <= 1e-13
    assert abs(got[0].sum() - h.sum()) <= 1e-12 * h.sum()


def test_walls_keep_the_mass_full_size(gpu, warmed):
    """The warmed, moving flood between four walls, forcings off: 20 steps
    keep the total depth to 1e-12 (the moisture floor only clamps films
    that are already at the dry threshold)."""
    sim, _, _ = gpu
    s = warmed
    cfg = sim.SimulationConfig(cfl=s.cfl, max_dt=s.max_dt)
    with sim.Simulation(sim.Mesh2D(s.bed, s.dx, s.dy, s.manning), (s.h, s.hu, s.hv),
                        cfg) as sm:
        sm.run_steps(20)
        got = sm.states()
    assert np.all(np.isfinite(got[0]))
    assert abs(got[0].sum() - s.h.sum()) <= 1e-12 * s.h.sum()
