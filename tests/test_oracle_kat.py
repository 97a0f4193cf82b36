"""Known-answer tests of the CPU oracle, restated from the reference's own
unit tests (file:line cited per test). These pin the oracle where the
reference has closed forms or invariants; the golden-vector test pins it
against the reference's committed outputs."""
import math

import numpy as np
import pytest

from hydroflux_b200 import abi
from tests import cases

G = 9.81
W = (abi.HF_BC_WALL, 0.0)
TR = (abi.HF_BC_TRANSMISSIVE, 0.0)
WALLS = abi.make_boundaries(W, W, W, W)
TRANS = abi.make_boundaries(TR, TR, TR, TR)


def approx(a, b, eps):
    # approx::assert_relative_eq!(a, b, epsilon = eps): |a-b| <= eps or relative
    return abs(a - b) <= eps or abs(a - b) <= eps * max(abs(a), abs(b))


# ---------------------------------------------------------------- riemann.rs
@pytest.mark.parametrize("x_dir", [True, False])
def test_hllc_consistency(oracle, x_dir):  # riemann.rs:215-233
    u = np.array([1.5, 0.6, -0.3])
    f = oracle.hllc_flux(x_dir, u, u)
    h, hu, hv = u
    if x_dir:
        phys = [hu, hu * hu / h + h * h * 0.5 * G, hu * hv / h]
    else:
        phys = [hv, hv * hu / h, hv * hv / h + h * h * 0.5 * G]
    for a, b in zip(f, phys):
        assert approx(a, b, 1e-12)


def test_hllc_dry_dry_zero(oracle):  # riemann.rs:236-240
    z = np.zeros(3)
    assert np.all(oracle.hllc_flux(True, z, z) == 0.0)
    assert np.all(oracle.hllc_flux(False, z, z) == 0.0)


def test_hllc_dam_break_positive_and_supercritical(oracle):  # riemann.rs:243-284
    assert oracle.hllc_flux(True, [2.0, 0, 0], [0.5, 0, 0])[0] > 0
    assert oracle.hllc_flux(False, [2.0, 0, 0], [0.5, 0, 0])[0] > 0
    s = np.array([1.0, 10.0, 1.0])
    f = oracle.hllc_flux(True, s, s)
    assert approx(f[0], 10.0, 1e-12) and approx(f[1], 100.0 + 0.5 * G, 1e-12)


def test_hllc_tangential_velocity_through_contact(oracle):  # riemann.rs:287-310
    v = 2.5
    f = oracle.hllc_flux(True, [2.0, 0.0, 2.0 * v], [0.5, 0.0, 0.5 * v])
    assert f[0] > 0 and approx(f[2], f[0] * v, 1e-10)
    u = -1.3
    f = oracle.hllc_flux(False, [2.0, 2.0 * u, 0.0], [0.5, 0.5 * u, 0.0])
    assert f[0] > 0 and approx(f[1], f[0] * u, 1e-10)


def test_hllc_dry_bed_closed_form(oracle):  # riemann.rs:363-389
    c_l = math.sqrt(G)
    f = oracle.hllc_flux(True, [1.0, 0, 0], [0, 0, 0])
    assert approx(f[0], 2.0 / 3.0 * c_l, 1e-12)
    assert f[0] > 0.5 * c_l
    f = oracle.hllc_flux(True, [0, 0, 0], [1.0, 0, 0])  # riemann.rs:340-360
    assert f[0] < 0 and abs(f[0]) < 2.0 * c_l


def test_hllc_lake_at_rest_face(oracle):  # riemann.rs:391-402
    f = oracle.hllc_flux(True, [2.0, 0, 0], [2.0, 0, 0])
    assert approx(f[0], 0.0, 1e-12) and approx(f[1], 0.5 * G * 4.0, 1e-12)


def test_hllc_dual_matches_fd(oracle):  # riemann.rs:428-471
    ur = np.array([0.5, 0, 0])
    fd = (oracle.hllc_flux(True, [2.0 + 1e-5, 0, 0], ur)[0]
          - oracle.hllc_flux(True, [2.0 - 1e-5, 0, 0], ur)[0]) / 2e-5
    _, ad = oracle.dual_hllc_mass(False, [2.0, 0, 0], ur)
    assert approx(ad, fd, 1e-7)
    fd = (oracle.hllc_flux(True, [0, 0, 0], [1.0 + 1e-5, 0, 0])[0]
          - oracle.hllc_flux(True, [0, 0, 0], [1.0 - 1e-5, 0, 0])[0]) / 2e-5
    _, ad = oracle.dual_hllc_mass(True, [0, 0, 0], [1.0, 0, 0])
    assert approx(ad, fd, 1e-7)


# --------------------------------------------------------------- boundary.rs
FLAT = np.full((3, 3), 10.0)
Y_SLOPED = np.array([[0.0] * 3, [-0.01] * 3, [-0.02] * 3, [-0.03] * 3])
X_SLOPED = np.array([[0.0, -0.01, -0.02, -0.03]] * 2)


def test_ghost_transmissive_and_wall(oracle):  # boundary.rs:412-439
    u = np.array([1.5, 0.6, -0.3])
    for side in range(4):
        g, _ = oracle.ghost_cell(FLAT, None, 1, 1, abi.HF_BC_TRANSMISSIVE, 0, side, 0, u)
        assert np.array_equal(g, u)
    g, _ = oracle.ghost_cell(FLAT, None, 1, 1, abi.HF_BC_WALL, 0, 2, 1, u)
    assert np.array_equal(g, [1.5, -0.6, -0.3])
    g, _ = oracle.ghost_cell(FLAT, None, 1, 1, abi.HF_BC_WALL, 0, 1, 1, u)
    assert np.array_equal(g, [1.5, 0.6, 0.3])


def test_ghost_discharge_and_depth(oracle):  # boundary.rs:442-479
    inner = np.array([0.6, 1.2, 0.4])
    g, _ = oracle.ghost_cell(X_SLOPED, None, 1, 1, abi.HF_BC_DISCHARGE, 0.8, 2, 0, inner)
    assert np.allclose(g, [0.6, 0.8, 0.4], atol=1e-12)
    g, _ = oracle.ghost_cell(Y_SLOPED, None, 1, 1, abi.HF_BC_DISCHARGE, 0.7, 0, 0, inner)
    assert np.allclose(g, [0.6, 1.2, 0.7], atol=1e-12)
    g, _ = oracle.ghost_cell(Y_SLOPED, None, 1, 1, abi.HF_BC_DEPTH, 0.45, 1, 2, inner)
    assert np.allclose(g, [0.45, 1.2, 0.4], atol=1e-12)


def test_ghost_beds(oracle):  # boundary.rs:482-527
    inner = np.array([0.5, 0.0, 0.0])
    _, z = oracle.ghost_cell(Y_SLOPED, None, 1, 1, abi.HF_BC_TRANSMISSIVE, 0, 0, 1, inner)
    assert z == Y_SLOPED[0, 1]
    _, z = oracle.ghost_cell(Y_SLOPED, None, 1, 1, abi.HF_BC_WALL, 0, 1, 2, inner)
    assert z == Y_SLOPED[3, 2]
    _, z = oracle.ghost_cell(Y_SLOPED, None, 1, 1, abi.HF_BC_DISCHARGE, 1.0, 0, 1, inner)
    assert approx(z, 0.01, 1e-12)
    _, z = oracle.ghost_cell(Y_SLOPED, None, 1, 1, abi.HF_BC_DEPTH, 0.5, 1, 1, inner)
    assert approx(z, -0.04, 1e-12)
    _, z = oracle.ghost_cell(X_SLOPED, None, 1, 1, abi.HF_BC_DISCHARGE, 1.0, 2, 0, inner)
    assert approx(z, 0.01, 1e-12)
    _, z = oracle.ghost_cell(X_SLOPED, None, 1, 1, abi.HF_BC_DEPTH, 0.5, 3, 1, inner)
    assert approx(z, -0.04, 1e-12)


def test_ghost_discharge_on_dry_uses_manning_normal_depth(oracle):  # boundary.rs:193-219
    z = np.array([[0.0, -0.01, -0.02, -0.03]] * 2)
    n = np.full_like(z, 0.03)
    g, _ = oracle.ghost_cell(z, n, 1.0, 1.0, abi.HF_BC_DISCHARGE, 2.0, 2, 0, [0.0, 0.0, 0.0])
    assert approx(g[0], (0.03 * 2.0 / math.sqrt(0.01)) ** 0.6, 1e-12)
    g, _ = oracle.ghost_cell(np.zeros((2, 4)), n, 1.0, 1.0, abi.HF_BC_DISCHARGE, 2.0, 2, 0,
                             [0.0, 0.0, 0.0])
    assert g[0] == 0.0  # flat: no override


# ----------------------------------------------------------------- source.rs
def test_friction_closed_form(oracle):  # source.rs:261-279
    n = np.full((1, 1), 0.04)
    h, hu, hv = oracle.manning_friction_step(n, [[1.0]], [[2.0]], [[1.0]], 0.05, 1e-9)
    speed = math.sqrt(5.0)
    factor = 1.0 + 0.05 * G * 0.04 * 0.04 * speed / 1.0 ** (4.0 / 3.0)
    assert approx(hu[0, 0], 2.0 / factor, 1e-12) and approx(hv[0, 0], 1.0 / factor, 1e-12)
    assert h[0, 0] == 1.0


def test_friction_invariants(oracle):  # source.rs:181-258, 281-305, 392-409
    st = (np.array([[1.0, 2.0]]), np.array([[2.0, -1.5]]), np.array([[-0.5, 0.7]]))
    out = oracle.manning_friction_step(np.zeros((1, 2)), *st, 0.1, 1e-9)
    assert all(np.array_equal(a, b) for a, b in zip(out, st))  # zero n identity
    out = oracle.manning_friction_step(np.full((3, 4), 0.03), np.full((3, 4), 2.0),
                                       np.zeros((3, 4)), np.zeros((3, 4)), 0.1, 1e-9)
    assert np.all(out[1] == 0) and np.all(out[2] == 0) and np.all(out[0] == 2.0)
    out = oracle.manning_friction_step(np.full((1, 2), 0.03), [[0.0, 0.0]], [[0.0, 1e-30]],
                                       [[0.0, -1e-30]], 0.1, 1e-9)
    assert out[1][0, 1] == 1e-30 and out[2][0, 1] == -1e-30  # dry untouched
    h, hu, hv = [[1.0]], [[2.0]], [[1.0]]
    ang0 = math.atan2(1.0, 2.0)
    for _ in range(50):
        h, hu, hv = oracle.manning_friction_step(np.full((1, 1), 0.05), h, hu, hv, 0.1, 1e-9)
        assert approx(math.atan2(hv[0, 0], hu[0, 0]), ang0, 1e-12)
    h, hu, hv = [[1.5]], [[3.0]], [[0.0]]
    for _ in range(20):
        h, hu, hv = oracle.manning_friction_step(np.full((1, 1), 0.04), h, hu, hv, 0.05, 1e-9)
        assert hv[0, 0] == 0.0 and hu[0, 0] > 0


def test_friction_dual_matches_fd(oracle):  # source.rs:420-473
    def hu_of_n(nv):
        return oracle.manning_friction_step(np.full((1, 1), nv), [[1.0]], [[3.0]], [[0.0]],
                                            0.1, 1e-9)[1][0, 0]
    fd = (hu_of_n(0.04 + 1e-5) - hu_of_n(0.04 - 1e-5)) / 2e-5
    _, ad = oracle.dual_friction_hu(False, 1.0, 3.0, 0.0, 0.04, 0.1, 1e-9)
    assert approx(ad, fd, 1e-7)

    def hu_of_h(hv_):
        return oracle.manning_friction_step(np.full((1, 1), 0.04), [[hv_]], [[hv_ * 2.0]],
                                            [[hv_ * -1.0]], 0.1, 1e-9)[1][0, 0]
    fd = (hu_of_h(1.5 + 1e-5) - hu_of_h(1.5 - 1e-5)) / 2e-5
    _, ad = oracle.dual_friction_hu(True, 1.5, 2.0, -1.0, 0.04, 0.1, 1e-9)
    assert approx(ad, fd, 1e-6)


def test_point_sources(oracle):  # source.rs:479-577
    z3 = np.zeros((3, 3))
    h, hu, hv = oracle.apply_point_sources(z3, z3, z3, [(1, 1, 2.0)], 0.5, 1.0, 1.0)
    assert approx(h[1, 1], 1.0, 1e-12) and h.sum() == h[1, 1] and hu[1, 1] == 0
    h, hu, hv = np.zeros((1, 1)), np.zeros((1, 1)), np.zeros((1, 1))
    for _ in range(10):
        h, hu, hv = oracle.apply_point_sources(h, hu, hv, [(0, 0, 1.0)], 0.1, 1.0, 1.0)
    assert approx(h[0, 0], 1.0, 1e-12)
    a = oracle.apply_point_sources(*(np.zeros((1, 1)),) * 3, [(0, 0, 1.0)], 1.0, 1.0, 1.0)[0]
    b = oracle.apply_point_sources(*(np.zeros((1, 1)),) * 3, [(0, 0, 1.0)], 1.0, 2.0, 2.0)[0]
    assert approx(a[0, 0], 4.0 * b[0, 0], 1e-12)
    h, hu, hv = oracle.apply_point_sources([[1.0]], [[5.0]], [[0.0]], [(0, 0, -10.0)], 1.0, 1.0,
                                           1.0)
    assert h[0, 0] == 0.0 and hu[0, 0] == 0.0 and hv[0, 0] == 0.0
    z2 = np.zeros((2, 2))
    h, _, _ = oracle.apply_point_sources(z2, z2, z2, [(0, 0, 1.0), (1, 1, 2.0)], 1.0, 1.0, 1.0)
    assert approx(h[0, 0], 1.0, 1e-12) and approx(h[1, 1], 2.0, 1e-12) and h[0, 1] == 0


def test_rain(oracle):  # source.rs:583-639
    z = np.zeros((3, 4))
    h, hu, hv = oracle.apply_rain(z, z, z, 0.001, 60.0)
    assert np.allclose(h, 0.06, atol=1e-12) and np.all(hu == 0)
    h, hu, hv = oracle.apply_rain([[1.0]], [[3.0]], [[-1.5]], 0.005, 4.0)
    assert approx(h[0, 0], 1.02, 1e-12) and hu[0, 0] == 3.0 and hv[0, 0] == -1.5
    h, hu, hv = oracle.apply_rain([[0.01]], [[0.5]], [[0.0]], -1.0, 1.0)
    assert h[0, 0] == 0 and hu[0, 0] == 0
    h, hu, hv = oracle.apply_rain([[1.0]], [[0.5]], [[-0.3]], 0.0, 100.0)
    assert h[0, 0] == 1.0 and hu[0, 0] == 0.5
    h, hu, hv = np.zeros((1, 1)), np.zeros((1, 1)), np.zeros((1, 1))
    for _ in range(360):
        h, hu, hv = oracle.apply_rain(h, hu, hv, 0.01 / 3600.0, 1.0)
    assert approx(h[0, 0], 0.001, 1e-12)


# ----------------------------------------------------------------- update.rs
def test_wave_speeds_and_dry_cfl(oracle):  # update.rs:1369-1391
    z = np.zeros((4, 5))
    assert oracle.max_wave_speeds(z, z, z) == (0.0, 0.0)
    assert oracle.cfl_time_step(z, 1, 1, z, z, z, 0.5) == math.inf
    h = np.zeros((2, 2)); hu = np.zeros((2, 2)); hv = np.zeros((2, 2))
    h[0, 0], hu[0, 0], hv[0, 0] = 1.0, 2.0, 3.0
    sx, sy = oracle.max_wave_speeds(h, hu, hv)
    assert approx(sx, 2.0 + math.sqrt(G), 1e-12) and approx(sy, 3.0 + math.sqrt(G), 1e-12)


def _loop(O, z, dx, dy, h, hu, hv, bcs, nsteps, ssprk=False, cfl=0.4):
    for _ in range(nsteps):
        dt = O.cfl_time_step(z, dx, dy, h, hu, hv, cfl)
        if not math.isfinite(dt):
            break
        step = O.ssprk2_step if ssprk else O.forward_euler_step
        h, hu, hv = step(z, dx, dy, h, hu, hv, bcs, dt)
    return h, hu, hv


def test_lake_at_rest_flat_exact(oracle):  # update.rs:1394-1410, 1834-1851
    z = np.zeros((10, 12))
    for step in (oracle.forward_euler_step, oracle.ssprk2_step):
        h, hu, hv = np.full((10, 12), 2.0), np.zeros((10, 12)), np.zeros((10, 12))
        for _ in range(100):
            h, hu, hv = step(z, 1, 1, h, hu, hv, TRANS, 0.01)
        assert np.allclose(h, 2.0, atol=1e-12) and np.allclose(hu, 0, atol=1e-12)


BEDS = {
    "x": lambda: np.repeat((-(np.arange(30) * 0.05))[None, :], 6, 0),  # update.rs:1413
    "y": lambda: np.repeat((-(np.arange(30) * 0.05))[:, None], 6, 1),  # update.rs:1435
    "diag": lambda: -(np.arange(20)[None, :] * 0.03) - (np.arange(15)[:, None] * 0.04),  # 1458
    "bumpy": lambda: cases.gaussian_bed(20, 20, 1.5),  # update.rs:1482
}


@pytest.mark.parametrize("bed", list(BEDS))
@pytest.mark.parametrize("ssprk", [False, True])
def test_lake_at_rest_sloped(oracle, bed, ssprk):  # update.rs:1412-1500, 1853-1873
    if ssprk and bed not in ("diag",):
        pytest.skip("reference checks SSP-RK2 lake-at-rest on the diagonal bed")
    z = BEDS[bed]()
    eta = 3.0 if bed == "bumpy" else 5.0
    h0 = eta - z
    h, hu, hv = _loop(oracle, z, 1, 1, h0, 0 * z, 0 * z, WALLS, 200, ssprk)
    assert np.allclose(h, h0, atol=1e-10, rtol=1e-10)
    assert np.abs(hu).max() <= 1e-10 and np.abs(hv).max() <= 1e-10


@pytest.mark.parametrize("kind", ["island", "bank"])
def test_lake_at_rest_shoreline(oracle, kind):  # update.rs:1523-1605
    if kind == "island":
        z = cases.gaussian_bed(21, 21, 2.5)
        eta = 1.0
    else:
        z = np.repeat((-0.5 + 2.0 * np.arange(30) / 29.0)[None, :], 4, 0)
        eta = 0.5
    h0 = np.maximum(eta - z, 0.0)
    h, hu, hv = _loop(oracle, z, 1, 1, h0, 0 * z, 0 * z, WALLS, 200)
    assert np.abs(h - h0).max() < 1e-10
    assert np.abs(hu).max() < 1e-10 and np.abs(hv).max() < 1e-10
    if kind == "island":
        assert approx(h0.sum(), h.sum(), 1e-12)


@pytest.mark.parametrize("ssprk", [False, True])
def test_mass_conserved_walls(oracle, ssprk):  # update.rs:1503-1520, 1876-1893
    z = np.zeros((25, 25))
    h0 = cases.gaussian_bump(25, 25)
    h, _, _ = _loop(oracle, z, 1, 1, h0, 0 * z, 0 * z, WALLS, 200, ssprk)
    assert approx(h0.sum(), h.sum(), 1e-10)


def test_draining_cell_regression(oracle):  # update.rs:1608-1644
    z = np.zeros((3, 3))
    h = np.zeros((3, 3)); hv = np.zeros((3, 3))
    h[0, 1], hv[0, 1] = 0.05, 0.25
    m0 = h.sum()
    h, hu, hv = oracle.forward_euler_step(z, 1, 1, h, 0 * z, hv, WALLS, 0.25)
    assert h[0, 1] <= abi.H_DRY and h[1, 1] > 0.025
    assert approx(m0, h.sum(), 1e-12)


def test_wetting_front_mass(oracle):  # update.rs:1690-1717
    z = np.zeros((30, 30))
    h0 = np.repeat(np.where(np.arange(30) < 15, 1.0, 0.0)[None, :], 30, 0)
    h, _, _ = _loop(oracle, z, 1, 1, h0, 0 * z, 0 * z, WALLS, 300)
    assert np.all(np.isfinite(h)) and np.all(h >= 0)
    assert approx(h0.sum(), h.sum(), 1e-12)


def test_thin_film_dt(oracle):  # update.rs:1720-1754
    z = np.zeros((4, 4))
    h = np.ones((4, 4)); hu = np.zeros((4, 4)); hv = np.zeros((4, 4))
    h[1, 1], hu[1, 1], hv[1, 1] = 1.1e-6, 1.0, 1.0
    dt = oracle.cfl_time_step(z, 1, 1, h, hu, hv, 0.4)
    assert dt > 0.9 * 0.4 / (2.0 * math.sqrt(G))
    h, hu, hv = oracle.forward_euler_step(z, 1, 1, h, hu, hv, WALLS, dt)
    if h[1, 1] > abi.H_VEL:
        assert max(abs(hu[1, 1] / h[1, 1]), abs(hv[1, 1] / h[1, 1])) < 10
    else:
        assert hu[1, 1] == 0 and hv[1, 1] == 0


@pytest.mark.parametrize("ssprk", [False, True])
def test_isotropy(oracle, ssprk):  # update.rs:1807-1826, 1896-1912
    z = np.zeros((21, 21))
    h, _, _ = _loop(oracle, z, 1, 1, cases.gaussian_bump(21, 21), 0 * z, 0 * z, TRANS, 50, ssprk)
    assert np.allclose(h, h[::-1, :], atol=1e-10)
    assert np.allclose(h, h.T, atol=1e-10)
    if not ssprk:
        assert np.allclose(h, h[:, ::-1], atol=1e-10)


def test_ssprk2_positivity_at_dry_interface(oracle):  # update.rs:1915-1941
    z = np.zeros((3, 100))
    h0 = np.repeat(np.where(np.arange(100) < 50, 1.0, 0.0)[None, :], 3, 0)
    h, hu, hv = _loop(oracle, z, 1, 1, h0, 0 * z, 0 * z, TRANS, 300, True)
    assert np.all(np.isfinite(h)) and np.all(h >= 0) and np.all(np.isfinite(hu))


def test_dual_mass_derivatives(oracle):  # update.rs:1954-2038
    m, dm = oracle.dual_mass_step(4, 5, 1.0, 1.0, False, 2.0, 0.0, False, abi.HF_BC_WALL, 0.01)
    assert approx(m, 40.0, 1e-10) and approx(dm, 20.0, 1e-10)
    m, dm = oracle.dual_mass_step(6, 6, 1.0, 1.0, True, 0.5, 3.0, True, abi.HF_BC_WALL, 0.005)
    assert approx(dm, -36.0, 1e-8)


# -------------------------------------------------------------------- sim.rs
def _bump(n):  # sim.rs:279-288
    x = np.arange(n) - n / 2.0
    X, Y = np.meshgrid(x, x)
    return 1.0 + 0.3 * np.exp(-(X * X + Y * Y) / 8.0)


def test_driver_matches_hand_loop_bitwise(oracle):  # sim.rs:290-321
    z = np.zeros((16, 16)); n = np.full((16, 16), 0.03)
    h0 = _bump(16)
    cfg = abi.make_config()
    r = oracle.sim_run(z, n, 1.0, 1.0, h0, 0 * z, 0 * z, cfg, 2.0)
    assert r["status"] == 0
    h, hu, hv = h0, 0 * z, 0 * z
    t = 0.0
    while t < 2.0:
        dt = min(oracle.cfl_time_step(z, 1, 1, h, hu, hv, 0.4, bcs=WALLS, n=n), 60.0, 2.0 - t)
        h, hu, hv = oracle.ssprk2_step(z, 1, 1, h, hu, hv, WALLS, dt, n)
        h, hu, hv = oracle.manning_friction_step(n, h, hu, hv, dt, abi.H_DRY)
        t += dt
    assert r["t"] == t
    assert np.array_equal(r["h"], h) and np.array_equal(r["hu"], hu) and np.array_equal(r["hv"], hv)


def test_driver_mass_and_errors(oracle):  # sim.rs:323-373
    z = np.zeros((20, 20))
    h0 = _bump(20)
    r = oracle.sim_run(z, np.full_like(z, 0.03), 1, 1, h0, 0 * z, 0 * z, abi.make_config(), 5.0)
    assert r["status"] == 0 and r["steps"] > 0 and approx(h0.sum(), r["h"].sum(), 1e-10)
    z8 = np.zeros((8, 8))
    r = oracle.sim_run(z8, None, 1, 1, _bump(8), 0 * z8, 0 * z8, abi.make_config(cfl=1.5), 1.0)
    assert r["status"] == abi.HF_ERR_INVALID_CONFIG
    r = oracle.sim_run(z8, None, 1, 1, _bump(8), 0 * z8, 0 * z8, abi.make_config(max_steps=3),
                       1e9)
    assert r["status"] == abi.HF_ERR_STEP_BUDGET and r["steps"] == 3
    # Dry domain: dt = min(inf, max_dt) is finite; a zero cap is degenerate.
    r = oracle.sim_step(z8, None, 1, 1, 0 * z8, 0 * z8, 0 * z8, abi.make_config(), 0.0)
    assert r["status"] == abi.HF_ERR_DEGENERATE_DT


def test_series_eval(oracle):
    t = [0.0, 10.0, 10.0, 20.0]
    v = [0.0, 1.0, 5.0, 5.0]
    assert oracle.series_eval(t, v, -1.0) == 0.0
    assert oracle.series_eval(t, v, 5.0) == 0.5
    assert oracle.series_eval(t, v, 10.0) == 5.0  # equal stamps: a step
    assert oracle.series_eval(t, v, 30.0) == 5.0


# ------------------------------------------------------ pow as the libm rounds it
POW_EXPONENTS = (4.0 / 3.0, 3.0 / 5.0, 4.0 / 3.0 - 1.0, 3.0 / 5.0 - 1.0)


def _pow_samples(rng, n):
    """Depth-like values (log-uniform 1e-14 .. 1e6), values within 2^-29 of
    1, and random bit patterns over every positive double (subnormals,
    the overflow / underflow branches, inf and NaN)."""
    depth = np.exp(rng.uniform(np.log(1e-14), np.log(1e6), n))
    near1 = 1.0 + rng.integers(-(1 << 23), 1 << 23, n) * 2.0 ** -52
    bits = (rng.integers(0, 1 << 63, n, dtype=np.uint64)).view(np.float64)
    return np.concatenate([depth, near1, np.abs(bits), [0.0, -0.0, 1.0, np.inf, -np.inf,
                                                        np.nan, -1.0, 5e-324, 1.7e308]])


@pytest.mark.parametrize("y", POW_EXPONENTS)
def test_pow_restatement_matches_host_libm(oracle, y):
    """hf_pow.h's pow (what the GPU runs) equals the host C library's pow
    (what the reference's f64::powf calls) bit for bit: the step's two
    exponents and the Dual's n - 1, on 3 x 10^6 inputs each."""
    rng = np.random.default_rng(abs(int(y * 1e6)))
    n, first = oracle.pow_mismatches(_pow_samples(rng, 1_000_000), y)
    assert n == 0, f"x^{y!r}: {n} mismatches, e.g. {[float.hex(float(v)) for v in first]}"
    assert oracle.pow_port(0.0, y) == (0.0 if y > 0 else math.inf)
    assert math.isnan(oracle.pow_port(-1.0, y)) and oracle.pow_port(1.0, y) == 1.0


def test_pow_modes_agree_on_a_wetting_run(oracle):
    """Whole runs in the oracle's two pow modes (host libm, restatement)
    are identical bit for bit on a run that wets a dry valley with rain and
    an inflow (friction on every wet cell, thresholds crossed everywhere),
    and both keep every printed digit of the reference's MacDonald run."""
    import os

    from hydroflux_b200 import ensemble, workloads
    from tests.test_oracle_golden import run_free_loop
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_verif.npz"))
    s = workloads.valley(n=64, dx=5.0, seed=4, peak=60.0, t_end=600.0)
    out = {}
    try:
        for mode in ("libm", "port"):
            oracle.set_pow_mode(mode)
            r = oracle.sim_run(s.bed, s.manning, s.dx, s.dy, s.h, s.hu, s.hv,
                               ensemble.scenario_config(s), s.t_end,
                               forcing=workloads.oracle_forcing(s))
            assert r["status"] == 0
            c = cases.macdonald()
            h, _, _ = run_free_loop(oracle, c)
            assert np.array_equal(cases.golden_profile(c, h), golden["macdonald"])
            out[mode] = r
    finally:
        oracle.set_pow_mode("libm")
    assert out["libm"]["steps"] == out["port"]["steps"] > 50
    for k in ("h", "hu", "hv"):
        assert np.array_equal(out["libm"][k].view(np.uint64), out["port"][k].view(np.uint64))


def test_max_depth_exceeds_relief_flags_a_finite_blow_up(oracle):  # sim.rs:376-386
    bed = np.repeat(np.arange(4, dtype=float)[:, None] * 32.0, 4, axis=1)  # 0..96 m
    assert not oracle.max_depth_exceeds_relief(np.full((4, 4), 5.0), bed, 3.0)
    assert oracle.max_depth_exceeds_relief(np.full((4, 4), 3000.0), bed, 3.0)


def test_max_depth_exceeds_relief_floors_a_near_flat_mesh(oracle):  # sim.rs:388-397
    bed = np.zeros((3, 3))
    assert not oracle.max_depth_exceeds_relief(np.full((3, 3), 2.0), bed, 3.0)
    assert oracle.max_depth_exceeds_relief(np.full((3, 3), 50.0), bed, 3.0)


def test_max_depth_exceeds_relief_fold_semantics(oracle):
    """The folds of sim.rs:263-265: NaN depths and beds are skipped, the
    depth max starts at 0 (all-negative or all-NaN depths give 0), and a
    relief below 1 m or NaN takes the 1 m floor (an all-NaN bed gives
    -inf - inf = -inf, an all-inf bed inf - inf = NaN, and NaN.max(1.0)
    is 1.0)."""
    bed = np.array([[0.0, np.nan], [4.0, 1.0]])
    h = np.array([[np.nan, 11.9], [-3.0, np.nan]])
    assert not oracle.max_depth_exceeds_relief(h, bed, 3.0)   # 11.9 <= 12
    h[0, 0] = 12.5
    assert oracle.max_depth_exceeds_relief(h, bed, 3.0)
    assert not oracle.max_depth_exceeds_relief(np.full((2, 2), np.nan), bed, 0.0)  # 0 > 0 is false
    assert oracle.max_depth_exceeds_relief(np.full((2, 2), 1.5), np.full((2, 2), np.nan), 1.0)
    assert oracle.max_depth_exceeds_relief(np.full((2, 2), 1.5), np.full((2, 2), np.inf), 1.0)
    inf_bed = np.array([[0.0, np.inf], [1.0, 2.0]])  # infinite relief
    assert not oracle.max_depth_exceeds_relief(np.full((2, 2), 1e300), inf_bed, 1.0)
