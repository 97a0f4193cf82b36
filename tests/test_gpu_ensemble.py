"""Ensembles (hf_batch_*): every scenario of a batch must end bit-identical
to solving it alone (hf_sim run_until) and to the oracle with the correctly
rounded pow; a failing scenario stops alone."""
import numpy as np
import pytest

from hydroflux_b200 import abi
from tests.gpu_util import assert_parity, exact_fraction

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hydroflux_b200 import ensemble, workloads
    return ensemble, workloads


def mixed_scenarios(workloads):
    """Uneven sizes (incl. ones smaller than a tile and non-multiples of the
    tile), every boundary kind, rain + inflow, different horizons."""
    out = []
    for k, (n, bcs, t_end) in enumerate([
            (9, ((0, 0.0),) * 4, 40.0),
            (37, ((1, 0.0), (0, 0.0), (1, 0.0), (0, 0.0)), 60.0),
            (64, ((0, 0.0),) * 4, 30.0),
            # Discharge/Depth sides feeding this dry hilly valley drive the CFL dt
            # down to ~1e-5 s (the oracle does the same): a short horizon.
            (50, ((1, 0.0), (3, 0.4), (2, 0.3), (1, 0.0)), 0.1),
            (100, ((0, 0.0),) * 4, 20.0)]):
        s = workloads.valley(n=n, dx=5.0, seed=40 + k, peak=30.0 + 10 * k, t_end=t_end)
        s.bcs = bcs
        s.max_dt = 5.0
        out.append(s)
    return out


def solve_alone(workloads, s):
    with workloads.simulation_for(s) as sim:
        sim.run_until(s.t_end)
        return sim.states(), sim.steps(), sim.time()


def test_ensemble_matches_separate_solves(gpu, oracle):
    ensemble, workloads = gpu
    scns = mixed_scenarios(workloads)
    with ensemble.Ensemble(scns) as ens:
        left = ens.run()
        assert left == 0
        for k, s in enumerate(scns):
            info = ens.info(k)
            assert info["status"] == 0 and info["t"] == s.t_end
            got = ens.states(k)
            ref, steps, t = solve_alone(workloads, s)
            assert info["steps"] == steps and info["t"] == t
            assert exact_fraction(got, ref) == 1.0, f"scenario {k}"
    # and against the oracle (host libm pow) for three of them (the 100 x
    # 100 one has interior tiles)
    oracle.set_pow_mode("libm")
    try:
        for k in (1, 3, 4):
            s = scns[k]
            r = oracle.sim_run(s.bed, s.manning, s.dx, s.dy, s.h, s.hu, s.hv,
                               ensemble.scenario_config(s), s.t_end,
                               forcing=workloads.oracle_forcing(s))
            assert r["status"] == 0
            with ensemble.Ensemble([s]) as one:
                one.run()
                got = one.states(0)
            assert_parity(got, (r["h"], r["hu"], r["hv"]))
            assert exact_fraction(got, (r["h"], r["hu"], r["hv"])) == 1.0
    finally:
        oracle.set_pow_mode("libm")


def test_ensemble_partial_runs_and_failure_isolation(gpu):
    ensemble, workloads = gpu
    scns = mixed_scenarios(workloads)[:3]
    with ensemble.Ensemble(scns, max_steps=5) as ens:
        left = ens.run(max_batch_steps=3)
        assert left == 3
        assert all(ens.info(k)["steps"] == 3 for k in range(3))
        left = ens.run()
        assert left == 0
        # every scenario needs more than 5 steps: each fails alone with a budget error
        for k in range(3):
            info = ens.info(k)
            assert info["status"] == abi.HF_ERR_STEP_BUDGET and info["steps"] == 5


@pytest.mark.parametrize("schedule", [0, 1, 2, 3])
def test_every_schedule_gives_the_same_results(gpu, schedule):
    """The autotuner's candidates (static / dynamic tile order, scenario order
    / largest first) all give each scenario its lone solve, bit for bit."""
    ensemble, workloads = gpu
    scns = mixed_scenarios(workloads)
    with ensemble.Ensemble(scns) as ens:
        ens.set_schedule(schedule)
        assert ens.run() == 0
        assert ens.schedule()[0] == schedule
        for k, s in enumerate(scns):
            ref, steps, t = solve_alone(workloads, s)
            info = ens.info(k)
            assert info["steps"] == steps and info["t"] == t
            assert exact_fraction(ens.states(k), ref) == 1.0, f"scenario {k}"


def test_autotuner_picks_a_schedule_and_changes_nothing(gpu):
    ensemble, workloads = gpu
    scns = mixed_scenarios(workloads)
    with ensemble.Ensemble(scns) as ens:
        assert ens.schedule()[0] == -1
        assert ens.run(max_batch_steps=7) >= 0   # too short to tune: schedule 0
        assert ens.schedule()[0] == -1
        ens.run()
        sched, ms = ens.schedule()
        assert sched in (0, 1, 2, 3) and np.all(ms > 0.0)
        assert ms[sched] == ms.min()
        for k, s in enumerate(scns):
            ref, _, _ = solve_alone(workloads, s)
            assert exact_fraction(ens.states(k), ref) == 1.0, f"scenario {k}"
        with pytest.raises(ValueError):
            ens.set_schedule(4)


@pytest.mark.parametrize("schedule", [0, 1])
def test_ensemble_on_32x32_tiles(gpu, schedule):
    """With a 352 x 352 scenario beside the small ones the ensemble has at
    least 100 tiles of 32 x 32 and runs its batched kernels on that geometry
    (the lone solves of the small scenarios run on 32 x 8 tiles): every
    scenario still equals its lone solve bit for bit, after the same steps."""
    ensemble, workloads = gpu
    scns = mixed_scenarios(workloads)
    big = workloads.valley(n=352, dx=5.0, seed=77, t_end=1e9)
    big.max_dt = 5.0
    scns.append(big)
    tiles32 = sum(-(-s.shape[0] // 32) * -(-s.shape[1] // 32) for s in scns)
    assert tiles32 >= 100
    with ensemble.Ensemble(scns) as ens:
        ens.set_schedule(schedule)
        ens.run(max_batch_steps=30)
        for k, s in enumerate(scns):
            info = ens.info(k)
            assert info["status"] == 0 and info["steps"] > 0
            with workloads.simulation_for(s) as sim:
                sim.run_steps(info["steps"], s.t_end)
                assert sim.steps() == info["steps"] and sim.time() == info["t"]
                assert exact_fraction(ens.states(k), sim.states()) == 1.0, f"scenario {k}"


@pytest.mark.parametrize("with_small", [True, False])
def test_ensemble_solo_scenarios(gpu, with_small):
    """Scenarios of at least 512 tiles of 32 x 32 (here 736 x 736 and
    768 x 768) leave the tile lists and run their stages as their own
    k_stage_pf launches; with no small scenario the lists are empty. Every
    scenario equals its lone solve bit for bit, over the same steps and to
    the horizon."""
    ensemble, workloads = gpu
    big = []
    for k, (n, t_end) in enumerate(((736, 20.0), (768, 1e9))):
        s = workloads.valley(n=n, dx=5.0, seed=90 + k, peak=200.0, t_end=t_end)
        s.max_dt = 5.0
        big.append(s)
    scns = (mixed_scenarios(workloads) if with_small else []) + big
    with ensemble.Ensemble(scns) as ens:
        ens.set_schedule(1)
        ens.run(max_batch_steps=40)
        for k, s in enumerate(scns):
            info = ens.info(k)
            assert info["status"] == 0 and info["steps"] > 0
            with workloads.simulation_for(s) as sim:
                sim.run_steps(info["steps"], s.t_end)
                assert sim.steps() == info["steps"] and sim.time() == info["t"]
                assert exact_fraction(ens.states(k), sim.states()) == 1.0, f"scenario {k}"
