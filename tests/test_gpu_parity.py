"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Every test runs the same seeded inputs through the GPU library and the
oracle and requires max relative error <= 1e-10 in h/hu/hv with identical wet
masks (gpu_util.assert_parity). The reference's own verification profiles are
also checked digit for digit on the GPU.
"""
import math
import os

import numpy as np
import pytest

from hydroflux_b200 import abi
from tests import cases
from tests.gpu_util import assert_parity, exact_fraction, to_dev, to_host

pytestmark = pytest.mark.gpu

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_verif.npz"))


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hydroflux_b200 import sim, step
    return sim, step


@pytest.fixture(autouse=True)
def libm_pow(oracle):
    """The kernels raise to 4/3 and 3/5 with a pow that rounds as the host
    libm does (hf_pow.h); the oracle calls that libm (its default mode), so
    every comparison below is bitwise against the reference's arithmetic."""
    oracle.set_pow_mode("libm")
    yield
    oracle.set_pow_mode("libm")


def bcs_obj(sim, pairs):
    return sim.Boundaries2D(*[sim.Boundary(k, v) for k, v in pairs])


def random_case(nr, nc, seed, wet=0.7, film=0.05, slope=0.02):
    rng = np.random.default_rng(seed)
    z = rng.uniform(-0.5, 0.5, (nr, nc)) + slope * np.arange(nc)[None, :]
    h = rng.uniform(0.05, 2.0, (nr, nc))
    r = rng.uniform(size=(nr, nc))
    h[r > wet] = 0.0
    h[(r > wet - film) & (r <= wet)] = rng.uniform(0.0, 2e-5, size=int(((r > wet - film) & (r <= wet)).sum()))
    hu = rng.normal(0, 0.5, (nr, nc)) * (h > 1e-5)
    hv = rng.normal(0, 0.5, (nr, nc)) * (h > 1e-5)
    n = rng.uniform(0.0, 0.08, (nr, nc))
    return z, n, h, hu, hv


# 20x68 has exactly one tile whose 4-cell halo just fits inside the grid (the
# interior-tile instantiation at its threshold on all four sides); 20x67 has
# none; 40x70 and 64x96 mix both kinds. 3x40000 and 40000x3 are thin grids of
# 1,250 and 5,000 tiles, every one of them on two sides.
SHAPES = [(1, 1), (1, 9), (9, 1), (2, 2), (3, 3), (5, 7), (16, 32), (17, 33), (33, 17),
          (20, 67), (20, 68), (40, 70), (64, 96), (3, 40000), (40000, 3)]
BC_SETS = {
    "walls": ((1, 0),) * 4,
    "trans": ((0, 0),) * 4,
    "mixed": ((1, 0), (0, 0), (1, 0), (0, 0)),
    "discharge_depth": ((1, 0), (1, 0), (2, 0.4), (3, 0.3)),
    "dry_inflow": ((2, -0.2), (3, 0.5), (2, 0.6), (0, 0)),
}


def bcs_valid(pairs, nr, nc):
    for side, (k, _) in enumerate(pairs):
        if k in (2, 3) and (nr if side < 2 else nc) < 2:
            return False
    return True


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}")
@pytest.mark.parametrize("bcname", list(BC_SETS))
@pytest.mark.parametrize("integrator", ["euler", "ssprk2"])
def test_step_parity_random(gpu, oracle, shape, bcname, integrator):
    sim, step = gpu
    nr, nc = shape
    pairs = BC_SETS[bcname]
    if not bcs_valid(pairs, nr, nc):
        pytest.skip("Discharge/Depth need two cells normal to the side")
    z, n, h, hu, hv = random_case(nr, nc, seed=nr * 1000 + nc)
    bcs_c = abi.make_boundaries(*pairs)
    mesh = step.DeviceMesh(z, 1.5, 0.75, n)
    ws = step.StepWorkspace2D(nr, nc)
    dh, dhu, dhv = to_dev(h, hu, hv)
    ref = (h, hu, hv)
    for it in range(4):
        dt_ref = oracle.cfl_time_step(z, 1.5, 0.75, *ref, 0.45, bcs=bcs_c, n=n)
        dt_gpu = step.cfl_time_step_with_bcs(dh, dhu, dhv, mesh, bcs_obj(sim, pairs), 0.45, ws)
        assert dt_gpu == dt_ref
        dt = min(dt_ref, 0.05) if math.isfinite(dt_ref) else 0.05
        if integrator == "euler":
            ref = oracle.forward_euler_step(z, 1.5, 0.75, *ref, bcs_c, dt, n)
            step.forward_euler_step(dh, dhu, dhv, mesh, bcs_obj(sim, pairs), dt, ws)
        else:
            ref = oracle.ssprk2_step(z, 1.5, 0.75, *ref, bcs_c, dt, n)
            step.ssprk2_step(dh, dhu, dhv, mesh, bcs_obj(sim, pairs), dt, ws)
        got = to_host(dh, dhu, dhv)
        assert_parity(got, ref, what=f"step {it}: ")
        # Every operation is IEEE-rounded on both sides, and pow rounds as
        # the host libm does: the GPU step is bit-exact.
        assert exact_fraction(got, ref) == 1.0, f"step {it}: not bit-exact"


@pytest.mark.parametrize("offset", [0, 1], ids=["aligned", "off16"])
@pytest.mark.parametrize("shape", [(40, 70), (64, 96), (20, 67)], ids=lambda s: f"{s[0]}x{s[1]}")
def test_step_parity_field_alignment(gpu, oracle, shape, offset):
    """The pipelined stage stages its inputs with 16-byte copies of column
    pairs when the column count is even and every field starts on a 16-byte
    boundary, and element by element otherwise. Fields that start 8 bytes
    into their buffers (offset 1) and odd column counts take the second
    path; both give the oracle's bits."""
    torch = pytest.importorskip("torch")
    sim, step = gpu
    nr, nc = shape
    z, n, h, hu, hv = random_case(nr, nc, seed=nr * 7 + nc)
    pairs = BC_SETS["mixed"]
    bcs_c = abi.make_boundaries(*pairs)

    def placed(a):
        buf = torch.zeros(nr * nc + 2, dtype=torch.float64, device="cuda")
        v = buf[offset:offset + nr * nc].view(nr, nc)
        v.copy_(torch.as_tensor(a, dtype=torch.float64, device="cuda"))
        assert v.data_ptr() % 16 == 8 * offset
        return v

    mesh = step.DeviceMesh(placed(z), 1.5, 0.75, placed(n))
    assert mesh.bed.data_ptr() % 16 == 8 * offset
    ws = step.StepWorkspace2D(nr, nc)
    dh, dhu, dhv = placed(h), placed(hu), placed(hv)
    ref = (h, hu, hv)
    for it in range(4):
        dt = min(oracle.cfl_time_step(z, 1.5, 0.75, *ref, 0.45, bcs=bcs_c, n=n), 0.05)
        ref = oracle.ssprk2_step(z, 1.5, 0.75, *ref, bcs_c, dt, n)
        step.ssprk2_step(dh, dhu, dhv, mesh, bcs_obj(sim, pairs), dt, ws)
        got = to_host(dh, dhu, dhv)
        assert exact_fraction(got, ref) == 1.0, f"step {it}: not bit-exact"


@pytest.mark.parametrize("shape", [(1, 1), (7, 5), (128, 96)])
def test_friction_rain_sources_parity(gpu, oracle, shape):
    sim, step = gpu
    nr, nc = shape
    z, n, h, hu, hv = random_case(nr, nc, seed=7 + nr)
    mesh = step.DeviceMesh(z, 2.0, 3.0, n)
    dh, dhu, dhv = to_dev(h, hu, hv)
    step.manning_friction_step(dh, dhu, dhv, mesh, 0.3, 1e-6)
    ref = oracle.manning_friction_step(n, h, hu, hv, 0.3, 1e-6)
    got = to_host(dh, dhu, dhv)
    assert_parity(got, ref)
    step.apply_rain(dh, dhu, dhv, -3e-3, 2.0)
    ref = oracle.apply_rain(*ref, -3e-3, 2.0)
    assert_parity(to_host(dh, dhu, dhv), ref)
    srcs = [(nr - 1, 0, 5.0), (0, nc - 1, -100.0), (nr // 2, nc // 2, 1.0), (nr // 2, nc // 2, 2.5)]
    step.apply_point_sources(dh, dhu, dhv, srcs, 0.7, 2.0, 3.0)
    ref = oracle.apply_point_sources(*ref, srcs, 0.7, 2.0, 3.0)
    got = to_host(dh, dhu, dhv)
    assert_parity(got, ref)
    assert np.array_equal(got[0], ref[0])


def test_hllc_known_answers(gpu, oracle):
    import torch
    sim, step = gpu
    states = [([1.5, 0.6, -0.3], [1.5, 0.6, -0.3]), ([1.0, 0, 0], [0, 0, 0]),
              ([0, 0, 0], [1.0, 0, 0]), ([2.0, 0, 5.0], [0.5, 0, 1.25]), ([0, 0, 0], [0, 0, 0]),
              ([1.0, 10.0, 1.0], [1.0, 10.0, 1.0]), ([2.0, 1.0, 0.5], [0.7, 0.3, -0.2]),
              ([1e-13, 1.0, 1.0], [0.3, -2.0, 0.1])]
    ul = torch.tensor([s[0] for s in states], dtype=torch.float64, device="cuda")
    ur = torch.tensor([s[1] for s in states], dtype=torch.float64, device="cuda")
    for x_dir in (True, False):
        out = step.hllc_flux(x_dir, ul, ur).cpu().numpy()
        for k, (a, b) in enumerate(states):
            assert np.array_equal(out[k], oracle.hllc_flux(x_dir, a, b)), (x_dir, k)
    out = step.hllc_flux(True, ul, ur).cpu().numpy()
    assert abs(out[1, 0] - 2.0 / 3.0 * math.sqrt(9.81)) <= 1e-12  # riemann.rs:363-389


@pytest.mark.parametrize("pow_mode", ["libm", "port"])
@pytest.mark.parametrize("builder", cases.VERIF_CASES, ids=lambda b: b.__name__)
def test_reference_profiles_on_gpu(gpu, oracle, builder, pow_mode):
    """The reference's verification runs, through the GPU free functions:
    bitwise against the oracle with the host libm's pow and with its
    restatement, and digit for digit against the reference's committed
    profiles."""
    sim, step = gpu
    oracle.set_pow_mode(pow_mode)
    c = builder()
    pairs = c["bcs"]
    mesh = step.DeviceMesh(c["z"], c["dx"], c["dy"], c["n"])
    ws = step.StepWorkspace2D(*c["z"].shape)
    dh, dhu, dhv = to_dev(c["h"], c["hu"], c["hv"])
    b = bcs_obj(sim, pairs)
    t = 0.0
    while t < c["t_end"]:
        dt = min(step.cfl_time_step(dh, dhu, dhv, mesh, c["cfl"], ws), c["t_end"] - t)
        step.ssprk2_step(dh, dhu, dhv, mesh, b, dt, ws)
        if c["friction"] is not None:
            step.manning_friction_step(dh, dhu, dhv, mesh, dt, c["friction"])
        t += dt
    got = to_host(dh, dhu, dhv)
    from tests.test_oracle_golden import run_free_loop
    ref = run_free_loop(oracle, c)
    assert_parity(got, ref)
    assert exact_fraction(got, ref) == 1.0
    assert np.array_equal(cases.golden_profile(c, got[0]), GOLDEN[c["golden"]])


@pytest.mark.parametrize("pow_mode", ["libm", "port"])
def test_dam_break_256_simulation(gpu, oracle, pow_mode):
    """Circular dam break 256x256 to t = 10 s through Simulation::run_until:
    bitwise against the oracle with the libm pow and with its restatement."""
    sim, step = gpu
    oracle.set_pow_mode(pow_mode)
    c = cases.dam_break_256()
    cfg = sim.SimulationConfig(cfl=c["cfl"], boundaries=sim.Boundaries2D.WALLS)
    mesh = sim.Mesh2D(c["z"], c["dx"], c["dy"], c["n"])
    with sim.Simulation(mesh, (c["h"], c["hu"], c["hv"]), cfg) as s:
        s.run_until(c["t_end"])
        got = s.states()
        t_gpu, n_gpu = s.time(), s.steps()
    r = oracle.sim_run(c["z"], c["n"], c["dx"], c["dy"], c["h"], c["hu"], c["hv"], cfg.to_c(),
                       c["t_end"])
    assert r["status"] == 0
    assert n_gpu == r["steps"]
    assert_parity(got, (r["h"], r["hu"], r["hv"]))
    assert t_gpu == r["t"]
    assert exact_fraction(got, (r["h"], r["hu"], r["hv"])) == 1.0
    assert abs(got[0].sum() - c["h"].sum()) <= 1e-10 * c["h"].sum()  # walls conserve mass


@pytest.mark.parametrize("integrator", [0, 1])
def test_simulation_forcing_parity(gpu, oracle, integrator):
    """Rain and a point-inflow hydrograph applied after every step at t_new."""
    sim, step = gpu
    nr, nc = 48, 70
    rng = np.random.default_rng(3)
    z = 0.01 * np.arange(nr)[:, None] + 0.05 * np.abs(np.arange(nc) - nc / 2)[None, :] \
        + rng.uniform(0, 0.05, (nr, nc))
    n = rng.choice([0.025, 0.035, 0.05, 0.08], size=(nr, nc))
    zeros = np.zeros((nr, nc))
    rain = ((0.0, 0.0), (5.0, 1e-3), (20.0, 1e-3), (20.0, 0.0))
    src_series = ((0.0, 0.0), (10.0, 4.0), (30.0, 0.0))
    bcs = sim.Boundaries2D(sim.Boundary.wall(), sim.Boundary.transmissive(),
                           sim.Boundary.transmissive(), sim.Boundary.wall())
    cfg = sim.SimulationConfig(cfl=0.5, integrator=sim.Integrator(integrator), boundaries=bcs,
                               max_dt=2.0)
    mesh = sim.Mesh2D(z, 5.0, 5.0, n)
    with sim.Simulation(mesh, (zeros, zeros, zeros), cfg) as s:
        s.set_rain(rain)
        s.set_point_sources([sim.PointSource(2, nc // 2, src_series),
                             sim.PointSource(2, nc // 2, 0.5)])
        s.run_until(40.0)
        got = s.states()
        steps = s.steps()
    from oracle.oracle import Forcing
    f = Forcing(rain=(np.array([p[0] for p in rain]), np.array([p[1] for p in rain])),
                sources=[(2, nc // 2, np.array([p[0] for p in src_series]),
                          np.array([p[1] for p in src_series])),
                         (2, nc // 2, np.array([0.0]), np.array([0.5]))])
    r = oracle.sim_run(z, n, 5.0, 5.0, zeros, zeros, zeros, cfg.to_c(), 40.0, forcing=f)
    assert r["status"] == 0 and steps == r["steps"]
    assert_parity(got, (r["h"], r["hu"], r["hv"]))
    # Wetting by rain and inflow crosses the H_DRY / H_VEL thresholds every
    # step; with pow rounded identically on both sides the runs stay bitwise.
    assert exact_fraction(got, (r["h"], r["hu"], r["hv"])) == 1.0


def test_simulation_step_and_errors(gpu, oracle):
    sim, step = gpu
    z = np.zeros((8, 8))
    x = np.arange(8) - 4.0
    h0 = 1.0 + 0.3 * np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / 8.0)
    zeros = np.zeros_like(z)
    mesh = sim.Mesh2D(z, 1.0, 1.0, 0.03)
    with sim.Simulation(mesh, (h0, zeros, zeros), sim.SimulationConfig(max_steps=3)) as s:
        dt = s.step(0.05)
        r = oracle.sim_step(z, np.full_like(z, 0.03), 1, 1, h0, zeros, zeros,
                            abi.make_config(max_steps=3), 0.05)
        assert dt == r["dt"] and s.steps() == 1
        assert_parity(s.states(), (r["h"], r["hu"], r["hv"]))
        with pytest.raises(sim.StepBudgetExhausted) as e:
            s.run_until(1e9)
        assert s.steps() == 4  # one step + a budget of three in run_until
        with pytest.raises(sim.DegenerateDt):
            s.step(0.0)
    with pytest.raises(sim.InvalidConfig):
        sim.Simulation(mesh, (h0, zeros, zeros), sim.SimulationConfig(cfl=1.5))
    with pytest.raises(sim.ShapeMismatch):
        sim.Simulation(mesh, (h0[:4], zeros, zeros))
    # The C ABI checks the Manning field itself (on the device after upload).
    import ctypes as C

    from hydroflux_b200._lib import lib
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    for bad in (-0.01, np.nan):
        n = np.full_like(z, 0.03)
        n[3, 5] = bad
        desc = abi.hf_mesh_desc(8, 8, 1.0, 1.0, dp(z), dp(n), 0.0)
        cfg = abi.make_config()
        hnd = C.c_void_p()
        rc = lib().hf_sim_create(C.byref(desc), dp(h0), dp(zeros), dp(zeros), C.byref(cfg), 0,
                                 C.byref(hnd))
        assert rc == abi.HF_ERR_INVALID_ARG and not hnd.value


def test_driver_matches_hand_loop_bitwise(gpu):
    """sim.rs:290-321 on the GPU: Simulation == hand-rolled free-function loop."""
    sim, step = gpu
    n = 16
    x = np.arange(n) - n / 2.0
    h0 = 1.0 + 0.3 * np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / 8.0)
    z = np.zeros((n, n))
    zeros = np.zeros_like(z)
    with sim.Simulation(sim.Mesh2D(z, 1.0, 1.0, 0.03), (h0, zeros, zeros)) as s:
        s.run_until(2.0)
        a = s.states()
        ta = s.time()
    mesh = step.DeviceMesh(z, 1.0, 1.0, 0.03)
    ws = step.StepWorkspace2D(n, n)
    dh, dhu, dhv = to_dev(h0, zeros, zeros)
    t = 0.0
    while t < 2.0:
        dt = min(step.cfl_time_step_with_bcs(dh, dhu, dhv, mesh, sim.Boundaries2D.WALLS, 0.4, ws),
                 60.0, 2.0 - t)
        step.ssprk2_step(dh, dhu, dhv, mesh, sim.Boundaries2D.WALLS, dt, ws)
        step.manning_friction_step(dh, dhu, dhv, mesh, dt, 1e-6)
        t += dt
    b = to_host(dh, dhu, dhv)
    assert ta == t
    assert all(np.array_equal(x_, y_) for x_, y_ in zip(a, b))


@pytest.mark.parametrize("bed", ["bumps", "shoreline"])
def test_lake_at_rest_and_mass_on_gpu(gpu, oracle, bed):
    """Still water over a rough, fully wet bed stays still to machine
    precision over 300 steps (the well-balanced property), bitwise equal to
    the oracle. With dry islands (a shoreline) the reference scheme itself
    develops small velocities at the wet/dry edges, so there only parity and
    mass (walls: conserved to 1e-12) are checked."""
    sim, _ = gpu
    nr, nc = 70, 90
    rng = np.random.default_rng(17)
    yy, xx = np.mgrid[0:nr, 0:nc]
    z = 0.3 * np.sin(xx / 7.0) * np.cos(yy / 5.0) + rng.uniform(0, 0.05, (nr, nc))
    eta = 0.25 if bed == "bumps" else 0.05
    if bed == "bumps":
        z = z - 0.6
    h = np.maximum(eta - z, 0.0)
    zero = np.zeros_like(h)
    cfg = sim.SimulationConfig(cfl=0.45, max_dt=0.5)
    with sim.Simulation(sim.Mesh2D(z, 1.0, 1.0, 0.03), (h, zero, zero), cfg) as s:
        s.run_steps(300)
        got = s.states()
    r = oracle.sim_run(z, np.full_like(z, 0.03), 1.0, 1.0, h, zero, zero, cfg.to_c(), 1e9,
                       stop_after=300)
    assert exact_fraction(got, (r["h"], r["hu"], r["hv"])) == 1.0
    if bed == "bumps":
        assert np.max(np.abs(got[1])) <= 1e-13 and np.max(np.abs(got[2])) <= 1e-13
        assert np.max(np.abs(got[0] + z - eta)) <= 1e-13
    assert abs(got[0].sum() - h.sum()) <= 1e-12 * h.sum()


def test_state_pool_reuse_and_release(gpu):
    """Handles created after others were destroyed reuse pooled memory and
    compute the same; releasing the pool's cache leaves live handles intact."""
    sim, _ = gpu
    from hydroflux_b200._lib import lib
    z, n, h, hu, hv = random_case(64, 96, 5)
    results = []
    live = sim.Simulation(sim.Mesh2D(z, 1.0, 1.0, n), (h, hu, hv))
    for k in range(3):
        with sim.Simulation(sim.Mesh2D(z, 1.0, 1.0, n), (h, hu, hv)) as s:
            s.run_steps(20)
            results.append(s.states())
        if k == 1:
            assert lib().hf_release_cached_memory(0) == 0
    live.run_steps(20)
    results.append(live.states())
    live.close()
    for r in results[1:]:
        assert all(np.array_equal(a, b) for a, b in zip(r, results[0]))


def test_free_functions_on_32x32_tiles_against_oracle(gpu, oracle):
    """The free-function entry points take the 32 x 32 tile geometry from
    100 such tiles on (here 352 x 330: 121 tiles, partial last tiles in both
    directions): cfl_time_step_with_bcs and ssprk2_step give the oracle's
    bits there too."""
    sim, step = gpu
    nr, nc = 352, 330
    z, n, h, hu, hv = random_case(nr, nc, seed=4242)
    pairs = BC_SETS["mixed"]
    bcs_c = abi.make_boundaries(*pairs)
    mesh = step.DeviceMesh(z, 1.5, 0.75, n)
    ws = step.StepWorkspace2D(nr, nc)
    dh, dhu, dhv = to_dev(h, hu, hv)
    ref = (h, hu, hv)
    for it in range(2):
        dt_ref = oracle.cfl_time_step(z, 1.5, 0.75, *ref, 0.45, bcs=bcs_c, n=n)
        dt_gpu = step.cfl_time_step_with_bcs(dh, dhu, dhv, mesh, bcs_obj(sim, pairs), 0.45, ws)
        assert dt_gpu == dt_ref
        dt = min(dt_ref, 0.05)
        ref = oracle.ssprk2_step(z, 1.5, 0.75, *ref, bcs_c, dt, n)
        step.ssprk2_step(dh, dhu, dhv, mesh, bcs_obj(sim, pairs), dt, ws)
        got = to_host(dh, dhu, dhv)
        assert exact_fraction(got, ref) == 1.0, f"step {it}: not bit-exact"
