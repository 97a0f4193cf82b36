"""Differentiation on the GPU (hf_tangent, hf_grad_manning).

* The DualD tangent reproduces the reference's published forward-mode
  calibration record (m1_inverse_manning_demo.rs; 12 Newton iterations).
* The tangent equals the oracle's Dual tangent over the same dt sequence:
  the misfit J bit for bit, dJ and the final tangent state to
  1e-10.
* The adjoint is the transpose of the tangent: for random directions in the
  Manning field and the initial state, dot(gradient, direction) equals the
  tangent's dJ; checkpoint intervals do not change the gradient (bit for
  bit) and repeated calls are bit-identical.
* Against central finite differences with the dt sequence frozen.
Problems cover open, wall, discharge (with the Manning normal-depth inflow
ghost on a dry bed) and depth boundaries, rain, point sources, wet/dry
fronts and both integrators.
"""
import os

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "reference_m1_inverse_manning.npz")


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hydroflux_b200 import calib, workloads
    return calib, workloads


@pytest.fixture(autouse=True)
def libm_pow(oracle):
    oracle.set_pow_mode("libm")
    yield


def m1_scenario(workloads, n_value):
    z, h, hu, hv = cases.m1_state()
    return workloads.Scenario("m1", z, np.full_like(z, n_value), 1.0, 1.0, h, hu, hv,
                              bcs=((1, 0.0), (1, 0.0), (0, 0.0), (0, 0.0)), cfl=0.4,
                              t_end=cases.M1_T_END, max_dt=1e9)


def test_tangent_matches_reference_newton_record(gpu):
    calib, workloads = gpu
    ones = np.ones((cases.M1_ROWS, cases.M1_COLS))
    with calib.Calibration(m1_scenario(workloads, cases.M1_N_TRUE), 5000) as cal:
        def centroid(n_value):
            cal.tangent(n_value * ones, dn=ones)
            st = cal.final_state()
            return cases.m1_centroid(st["h"][1], st["dh"][1])
        rows, _ = cases.m1_newton(centroid)
    cases.assert_matches_m1_record(rows, np.load(GOLDEN)["table"], dc=5e-12)


def lognormal(rng, shape, median=0.04, sigma=0.3):
    return median * np.exp(sigma * rng.standard_normal(shape))


def problem(workloads, name):
    """(scenario, n_steps, gauges)."""
    S = workloads.Scenario
    rng = np.random.default_rng(sum(map(ord, name)))
    if name == "valley":  # dry start, inflow + rain, open sides
        s = workloads.valley(n=48, dx=5.0, seed=3, peak=40.0, t_end=1e9)
        s.manning = lognormal(rng, s.shape)
        s.max_dt = 5.0
        return s, 120, np.array([5 * 48 + 24, 20 * 48 + 23, 30 * 48 + 25, 40 * 48 + 24])
    if name == "dambreak_fe":  # wet/dry dam break between walls, forward Euler, rain
        nr, nc = 24, 40
        x = np.arange(nc)[None, :] + 0.0 * np.arange(nr)[:, None]
        h = np.where(x < 12, 1.5, 0.0)
        z = 0.02 * x + 0.05 * np.sin(np.arange(nr))[:, None]
        s = S("dambreak_fe", z, lognormal(rng, (nr, nc)), 1.0, 1.0, h, np.zeros_like(h),
              np.zeros_like(h), bcs=((1, 0.0),) * 4, cfl=0.4, t_end=1e9, max_dt=1.0,
              rain=(np.array([0.0]), np.array([2e-4])), integrator=0)
        return s, 60, np.array([5 * nc + 14, 12 * nc + 20, 20 * nc + 8])
    if name == "inflow":  # discharge onto a dry slope (normal-depth ghost), depth outlet
        nr, nc = 20, 36
        x = np.arange(nc)[None, :] * np.ones((nr, 1))
        z = 2.0 - 0.02 * x + 0.1 * np.cos(0.7 * np.arange(nr))[:, None]
        h = np.zeros((nr, nc))
        s = S("inflow", z, lognormal(rng, (nr, nc)), 2.0, 2.0, h, h.copy(), h.copy(),
              bcs=((1, 0.0), (1, 0.0), (2, 0.6), (3, 0.05)), cfl=0.45, t_end=1e9, max_dt=0.5,
              sources=[(10, 20, np.array([0.0, 10.0, 40.0]), np.array([0.0, 2.0, 0.5]))])
        return s, 150, np.array([10 * nc + 3, 5 * nc + 12, 14 * nc + 30])
    if name == "wide":  # SSP-RK2 dam break whose front crosses interior tiles
        nr, nc = 40, 84
        x = np.arange(nc)[None, :] + 0.0 * np.arange(nr)[:, None]
        h = np.where(x < 40, 1.2, 0.0)
        z = 0.01 * x + 0.04 * np.sin(0.5 * np.arange(nr))[:, None]
        s = S("wide", z, lognormal(rng, (nr, nc)), 1.0, 1.0, h, np.zeros_like(h),
              np.zeros_like(h), bcs=((1, 0.0), (0, 0.0), (1, 0.0), (0, 0.0)), cfl=0.45,
              t_end=1e9, max_dt=1.0, rain=(np.array([0.0]), np.array([1e-4])))
        return s, 80, np.array([12 * nc + 36, 20 * nc + 44, 30 * nc + 50, 16 * nc + 60])
    raise KeyError(name)


# "wide" (40 x 84) has interior tiles, whose boundary branches are compiled
# out; the other grids are all edge tiles.
PROBLEMS = ["valley", "dambreak_fe", "inflow", "wide"]


def observations(cal, s, n_steps, G, seed):
    rng = np.random.default_rng(seed)
    _, gh, k = cal.run(s.manning * np.exp(0.2 * rng.standard_normal(s.shape)))
    obs = np.zeros((n_steps, G))
    obs[:k] = gh
    cal.set_observations(obs)
    return obs


def directions(rng, s):
    wet = s.h > 0
    return dict(dn=rng.standard_normal(s.shape) * 0.01,
                dh0=rng.standard_normal(s.shape) * 0.01 * wet,
                dhu0=rng.standard_normal(s.shape) * 0.01 * wet,
                dhv0=rng.standard_normal(s.shape) * 0.01 * wet)


@pytest.mark.parametrize("name", PROBLEMS)
def test_tangent_matches_oracle(gpu, oracle, name):
    calib, workloads = gpu
    s, K, gauges = problem(workloads, name)
    with calib.Calibration(s, K, gauges) as cal:
        obs = observations(cal, s, K, len(gauges), 1)
        d = directions(np.random.default_rng(2), s)
        J, dJ = cal.tangent(s.manning, **d)
        st = cal.final_state()
        dts = cal.dts()
    assert len(dts) == K
    ref = oracle.tangent_run(s.bed, s.manning, d["dn"], s.dx, s.dy, s.h, s.hu, s.hv,
                             workloads_config(s), dts, workloads.oracle_forcing(s),
                             dh=d["dh0"], dhu=d["dhu0"], dhv=d["dhv0"], gauges=gauges,
                             h_obs=obs.reshape(-1))
    assert J == ref["J"]
    assert np.array_equal(st["h"], ref["h"]) and np.array_equal(st["hu"], ref["hu"])
    assert abs(dJ - ref["dJ"]) <= 1e-10 * abs(ref["dJ"]) + 1e-300, (dJ, ref["dJ"])
    for k in ("dh", "dhu", "dhv"):
        scale = np.max(np.abs(ref[k]))
        assert np.max(np.abs(st[k] - ref[k])) <= 1e-10 * scale, k


def workloads_config(s):
    from hydroflux_b200.ensemble import scenario_config
    return scenario_config(s)


@pytest.mark.parametrize("name", PROBLEMS)
def test_adjoint_is_transpose_of_tangent(gpu, name):
    calib, workloads = gpu
    s, K, gauges = problem(workloads, name)
    with calib.Calibration(s, K, gauges, checkpoint_every=7) as cal:
        observations(cal, s, K, len(gauges), 3)
        J0, _, _ = cal.run(s.manning)
        J, g, (gh, ghu, ghv) = cal.gradient(s.manning, initial_state=True)
        assert J == J0
        assert np.all(np.isfinite(g)) and np.any(g != 0.0)
        rng = np.random.default_rng(4)
        for _ in range(4):
            d = directions(rng, s)
            _, dJ = cal.tangent(s.manning, **d)
            dot = (np.sum(g * d["dn"]) + np.sum(gh * d["dh0"]) + np.sum(ghu * d["dhu0"]) +
                   np.sum(ghv * d["dhv0"]))
            scale = (np.sum(np.abs(g * d["dn"])) + np.sum(np.abs(gh * d["dh0"])) +
                     np.sum(np.abs(ghu * d["dhu0"])) + np.sum(np.abs(ghv * d["dhv0"])))
            assert abs(dot - dJ) <= 1e-9 * max(abs(dJ), scale), (dot, dJ, scale)


def test_gradient_independent_of_checkpoints_and_deterministic(gpu):
    calib, workloads = gpu
    s, K, gauges = problem(workloads, "valley")
    grads = []
    for every in (1, 7, 45, 1000):
        with calib.Calibration(s, K, gauges, checkpoint_every=every) as cal:
            observations(cal, s, K, len(gauges), 5)
            grads.append(cal.gradient(s.manning)[1])
            if every == 7:
                assert np.array_equal(grads[-1], cal.gradient(s.manning)[1])
    for g in grads[1:]:
        assert np.array_equal(g, grads[0])


def test_gradient_against_central_differences(gpu):
    """Smooth, all-wet case; dt frozen to the base run (the gradient's dt)."""
    calib, workloads = gpu
    nr, nc = 32, 32
    xx, yy = np.meshgrid(np.arange(nc) + 0.5, np.arange(nr) + 0.5)
    h = 1.0 + 0.4 * np.exp(-((xx - 14) ** 2 + (yy - 17) ** 2) / 30.0)
    z = 0.01 * xx
    rng = np.random.default_rng(6)
    n = lognormal(rng, (nr, nc), median=0.05)
    s = workloads.Scenario("bump", z, n, 1.0, 1.0, h, np.zeros_like(h), np.zeros_like(h),
                           bcs=((0, 0.0),) * 4, cfl=0.4, t_end=1e9, max_dt=1.0)
    K, gauges = 40, np.array([5 * nc + 5, 16 * nc + 16, 25 * nc + 9])
    with calib.Calibration(s, K, gauges) as cal:
        obs = np.zeros((K, len(gauges)))
        obs[:] = 1.1
        cal.set_observations(obs)
        J, g = cal.gradient(n)
        for k in range(3):
            v = rng.standard_normal(n.shape)
            ad = float(np.sum(g * n * v))  # relative perturbation n (1 + eps v)
            # eps = 1e-6: J's rounding (~1e-15 |J|) over eps is ~1e-6 of dJ, and
            # the limiter's branch switches make J piecewise smooth, so a larger
            # eps does not help (1e-4 is off by ~3e-5); 2e-5 bounds both.
            eps = 1e-6
            Jp, _, _ = cal.run(n + eps * n * v, replay_dt=True)
            Jm, _, _ = cal.run(n - eps * n * v, replay_dt=True)
            fd = (Jp - Jm) / (2 * eps)
            assert abs(fd - ad) <= 2e-5 * abs(ad), (k, fd, ad)


def test_gradient_fd_converges_on_a_smooth_run(gpu):
    """Central differences converge to the adjoint to 1e-6 where the run is
    smooth: a 32 x 32 bump of water 1 to 1.4 m deep, all wet, 40 steps, no
    cell near the dry or velocity thresholds, dt frozen. At eps = 1e-5 (a
    relative perturbation of n) FD's truncation and J's rounding (about
    1e-15 |J| / eps) are both far below 1e-6."""
    calib, workloads = gpu
    nr = nc = 32
    K = 40
    xx, yy = np.meshgrid(np.arange(nc) + 0.5, np.arange(nr) + 0.5)
    h = 1.0 + 0.4 * np.exp(-((xx - nc * 0.45) ** 2 + (yy - nr * 0.53) ** 2) / (nr * 1.0))
    z = 0.01 * xx
    rng = np.random.default_rng(6)
    n = lognormal(rng, (nr, nc), median=0.05)
    s = workloads.Scenario("bump", z, n, 1.0, 1.0, h, np.zeros_like(h), np.zeros_like(h),
                           bcs=((0, 0.0),) * 4, cfl=0.4, t_end=1e9, max_dt=1.0)
    gauges = np.array([5 * nc + 5, (nr // 2) * nc + nc // 2, (nr - 7) * nc + 9])
    with calib.Calibration(s, K, gauges) as cal:
        obs = np.zeros((K, len(gauges)))
        obs[:] = 1.1
        cal.set_observations(obs)
        _, g = cal.gradient(n)
        for k in range(3):
            v = rng.standard_normal(n.shape)
            ad = float(np.sum(g * n * v))
            cal.run(n)  # the dt record of the base field
            eps = 1e-5
            Jp, _, _ = cal.run(n + eps * n * v, replay_dt=True)
            Jm, _, _ = cal.run(n - eps * n * v, replay_dt=True)
            fd = (Jp - Jm) / (2 * eps)
            assert abs(fd - ad) <= 1e-6 * abs(ad), (k, fd, ad)


def test_gradient_fd_on_the_calibration_problem(gpu):
    """The 512 x 512 valley misfit at 100 steps (the flood wetting the
    valley): FD agrees with the adjoint to 1e-4 at every eps from 1e-6 to
    1e-7, but no closer at any eps. The discrete step is discontinuous where
    a cell crosses the velocity floor (update.rs: momentum set to zero at
    h <= H_VEL) or the dry-cell paths, so J(n) has small jumps and central
    differences carry an error of ~1e-5 that does not shrink with eps; the
    adjoint is the derivative of the smooth pieces, the Dual's (it matches
    the tangent to 1e-13)."""
    calib, workloads = gpu
    K = 100
    P = workloads.calibration_problem(n=512, n_steps=K)
    s = P.scenario
    with calib.Calibration(s, K, P.gauges) as cal:
        _, gh, ko = cal.run(P.manning_true)
        ob = np.zeros((K, len(P.gauges)))
        ob[:ko] = gh
        cal.set_observations(ob)
        _, g = cal.gradient(s.manning)
        for d in range(3):
            v = np.random.default_rng(100 + d).standard_normal(s.shape) * s.manning
            ad = float(np.sum(g * v))
            cal.run(s.manning)
            for eps in (1e-6, 3e-7, 1e-7):
                Jp, _, _ = cal.run(s.manning + eps * v, replay_dt=True)
                Jm, _, _ = cal.run(s.manning - eps * v, replay_dt=True)
                fd = (Jp - Jm) / (2 * eps)
                assert abs(fd - ad) <= 1e-4 * abs(ad), (d, eps, fd, ad)


@pytest.mark.parametrize("name", PROBLEMS)
def test_tangent_lanes_equal_single_tangents(gpu, name):
    """Vector mode (DualN, autograd/src/dual_n.rs): every lane of one
    hf_tangent_lanes run equals hf_tangent along that direction bit for bit
    (dJ and the final tangent state), and the values equal a plain run."""
    calib, workloads = gpu
    s, K, gauges = problem(workloads, name)
    lanes = 5
    with calib.Calibration(s, K, gauges) as cal:
        observations(cal, s, K, len(gauges), 7)
        J0, _, _ = cal.run(s.manning)
        ref_state = cal.final_state()
        rng = np.random.default_rng(8)
        ds = [directions(rng, s) for _ in range(lanes)]
        stack = {k: np.stack([d[k] for d in ds]) for k in ds[0]}
        J, dJ = cal.tangent_lanes(s.manning, **stack)
        st = cal.final_state()
        lane_states = [cal.lane_state(l) for l in range(lanes)]
        assert J == J0
        for k in ("h", "hu", "hv"):
            assert np.array_equal(st[k], ref_state[k]), k
        for l, d in enumerate(ds):
            J1, dJ1 = cal.tangent(s.manning, **d)
            one = cal.final_state()
            assert J1 == J and dJ1 == dJ[l], (l, dJ1, dJ[l])
            for k in ("dh", "dhu", "dhv"):
                assert np.array_equal(lane_states[l][k], one[k]), (l, k)


def test_tangent_lanes_odd_steps_and_lane_counts(gpu):
    """Vector-mode runs replay CUDA graphs of an even number of steps, finish
    an odd count with one direct step, and keep one set of graphs per lane
    count: 75 steps (64 + 8 + 2 + 1) with the lane count changing between
    runs still equal the single tangents bit for bit, and the values equal
    a plain run."""
    calib, workloads = gpu
    s, _, gauges = problem(workloads, "inflow")
    K = 75
    with calib.Calibration(s, K, gauges) as cal:
        observations(cal, s, K, len(gauges), 11)
        cal.run(s.manning)
        ref = cal.final_state()
        rng = np.random.default_rng(12)
        ds = [directions(rng, s) for _ in range(4)]
        singles = []
        for d in ds:
            dJ1 = cal.tangent(s.manning, **d)[1]
            singles.append((dJ1, cal.final_state()))
        for lanes in (3, 1, 4, 3):
            stack = {k: np.stack([d[k] for d in ds[:lanes]]) for k in ds[0]}
            _, dJ = cal.tangent_lanes(s.manning, **stack)
            st = cal.final_state()
            for k in ("h", "hu", "hv"):
                assert np.array_equal(st[k], ref[k]), (lanes, k)
            for l in range(lanes):
                assert dJ[l] == singles[l][0], (lanes, l)
                one = cal.lane_state(l)
                for k in ("dh", "dhu", "dhv"):
                    assert np.array_equal(one[k], singles[l][1][k]), (lanes, l, k)


def test_tangent_lanes_zonal_gradient(gpu):
    """The forward-scaling use (solver-2d/examples/m1_forward_scaling.rs):
    P zonal Manning parameters in vertical stripes, all P derivatives in one
    vector-mode run; they equal the adjoint gradient summed over each zone."""
    calib, workloads = gpu
    s, K, gauges = problem(workloads, "valley")
    P = 8
    cols = np.arange(s.shape[1])
    zone = (cols * P) // s.shape[1]
    dn = np.stack([np.broadcast_to((zone == p).astype(float), s.shape) for p in range(P)])
    with calib.Calibration(s, K, gauges) as cal:
        observations(cal, s, K, len(gauges), 9)
        J, dJ = cal.tangent_lanes(s.manning, dn=dn)
        Jg, g = cal.gradient(s.manning)
        assert J == Jg
        for p in range(P):
            want = np.sum(g[:, zone == p])
            scale = np.sum(np.abs(g[:, zone == p]))
            assert abs(dJ[p] - want) <= 1e-9 * max(scale, abs(want)), (p, dJ[p], want)
        with pytest.raises(ValueError):
            cal.tangent_lanes(s.manning, dn=np.zeros((1025,) + s.shape))
        with pytest.raises(ValueError):
            cal.lane_state(P)
