"""Shared problem setups for the oracle and GPU parity tests.

Each builder restates a setup from the reference's own tests/examples (cited)
and returns a dict with the mesh (z, n, dx, dy), the initial SoA state
(h, hu, hv), the boundaries as four (kind, value) pairs (north, south, west,
east) and the loop parameters of the reference's free-function driver:
    while t < t_end: dt = min(cfl_time_step(cfl), t_end - t)
                     ssprk2_step(dt); [manning_friction_step(dt, dry_tol)]
"""
from __future__ import annotations

import math

import numpy as np

G = 9.81
T, W, Q, D = 0, 1, 2, 3  # boundary kinds


def stoker():
    """solver-2d/examples/gen_verification_data.rs:46-80 (dam break on dry bed)."""
    h_l, x_dam, length, t_end = 1.0, 50.0, 100.0, 4.0
    nc, nr = 400, 3
    dx = length / nc
    x = (np.arange(nc) + 0.5) * dx
    h = np.repeat(np.where(x < x_dam, h_l, 0.0)[None, :], nr, 0)
    z = np.zeros((nr, nc))
    return dict(name="stoker", z=z, n=np.zeros_like(z), dx=dx, dy=dx, h=h, hu=np.zeros_like(h),
                hv=np.zeros_like(h), bcs=((W, 0), (W, 0), (T, 0), (T, 0)), t_end=t_end,
                cfl=0.4, friction=None, golden="stoker", golden_row=nr // 2, decimals=6)


def macdonald():
    """gen_verification_data.rs:86-120 (uniform Manning flow, Discharge/Depth)."""
    q, slope, manning = 1.0, 0.01, 0.03
    h_n = (manning * q / math.sqrt(slope)) ** (3.0 / 5.0)
    nr, nc, dx = 5, 50, 1.0
    z = np.repeat((-(np.arange(nc) * dx * slope))[None, :], nr, 0)
    h = np.full((nr, nc), h_n)
    u = q / h_n
    c = math.sqrt(G * h_n)
    return dict(name="macdonald", z=z, n=np.full((nr, nc), manning), dx=dx, dy=dx, h=h,
                hu=np.full((nr, nc), q), hv=np.zeros((nr, nc)),
                bcs=((W, 0), (W, 0), (Q, q), (D, h_n)), t_end=2.0 * (nc * dx) / (u + c),
                cfl=0.4, friction=1e-9, golden="macdonald", golden_row=nr // 2, decimals=6)


def thacker():
    """gen_verification_data.rs:134-183 (planar oscillation in a paraboloid)."""
    h0, a, b = 0.1, 1.0, 0.1
    n = 80
    he = 1.25
    dx = 2.0 * he / n
    omega = math.sqrt(2.0 * G * h0) / a
    t_end = (2.0 * math.pi / omega) / 2.0
    xs = -he + (np.arange(n) + 0.5) * dx
    X, Y = np.meshgrid(xs, xs)
    z = h0 * ((X * X + Y * Y) / (a * a) - 1.0)
    u0 = -b * omega * math.sin(0.0)
    v0 = b * omega * math.cos(0.0)
    r2 = (X - b) ** 2 + Y ** 2
    h = np.maximum(h0 / (a * a) * (a * a - r2), 0.0)
    return dict(name="thacker", z=z, n=np.zeros_like(z), dx=dx, dy=dx, h=h, hu=h * u0,
                hv=h * v0, bcs=((W, 0),) * 4, t_end=t_end, cfl=0.4, friction=None,
                golden="thacker", golden_row=n // 2, decimals=6)


def uk_ea_t6():
    """gen_verification_data.rs:190-256 (urban dam break through buildings)."""
    buildings = [(150.0, 170.0, 20.0, 40.0), (150.0, 170.0, 60.0, 80.0),
                 (200.0, 220.0, 40.0, 60.0), (250.0, 270.0, 20.0, 40.0),
                 (250.0, 270.0, 60.0, 80.0), (320.0, 360.0, 35.0, 65.0)]
    nx, ny = 250, 50
    dx, dy = 500.0 / nx, 100.0 / ny
    X, Y = np.meshgrid((np.arange(nx) + 0.5) * dx, (np.arange(ny) + 0.5) * dy)
    inside = np.zeros_like(X, dtype=bool)
    for xa, xb, ya, yb in buildings:
        inside |= (X >= xa) & (X <= xb) & (Y >= ya) & (Y <= yb)
    z = np.where(inside, 5.0, 0.0)
    h = np.where(inside, 0.0, np.where(X < 100.0, 2.0, 0.0))
    return dict(name="uk_ea_t6", z=z, n=np.full_like(z, 0.03), dx=dx, dy=dy, h=h,
                hu=np.zeros_like(h), hv=np.zeros_like(h), bcs=((W, 0), (W, 0), (W, 0), (T, 0)),
                t_end=30.0, cfl=0.4, friction=1e-9, golden="uk_ea_t6", golden_row=None,
                decimals=5)


VERIF_CASES = [stoker, macdonald, thacker, uk_ea_t6]


def gaussian_bump(nr, nc, h_base=1.0, h_amp=0.5):
    """update.rs:1346-1367 (isotropy / mass tests)."""
    cx, cy = (nc - 1) / 2.0, (nr - 1) / 2.0
    w_sq = float(min(nr, nc)) ** 2 / 25.0
    j, i = np.meshgrid(np.arange(nc, dtype=float), np.arange(nr, dtype=float))
    return h_base + h_amp * np.exp(-((j - cx) ** 2 + (i - cy) ** 2) / w_sq)


def gaussian_bed(nr, nc, amp):
    """update.rs:1320-1335."""
    return gaussian_bump(nr, nc, 0.0, amp)


def dam_break_256():
    """Circular dam break on 256x256, dx = 1 m, flat bed, h = 10 m inside r < 50 m
    of the centre and 1 m outside, n = 0.03, walls, CFL 0.5, to t = 10 s."""
    n = 256
    xc = (np.arange(n) + 0.5)
    X, Y = np.meshgrid(xc, xc)
    r = np.sqrt((X - 128.0) ** 2 + (Y - 128.0) ** 2)
    h = np.where(r < 50.0, 10.0, 1.0)
    z = np.zeros((n, n))
    return dict(name="dam_break_256", z=z, n=np.full_like(z, 0.03), dx=1.0, dy=1.0, h=h,
                hu=np.zeros_like(h), hv=np.zeros_like(h), bcs=((W, 0),) * 4, t_end=10.0,
                cfl=0.5)


def golden_profile(case, h):
    if case["golden_row"] is None:
        return np.round(h.reshape(-1), case["decimals"])
    return np.round(h[case["golden_row"]], case["decimals"])


# ---------------------------------------------------------------------------
# Forward-mode calibration demo of the reference
# (solver-2d/examples/m1_inverse_manning_demo.rs:43-112): a 3 x 60 flat
# channel, dx = dy = 1, h = 1 m for j < 30 and 0.1 m beyond, at rest; walls
# north/south, transmissive west/east; uniform Manning n; SSP-RK2 with
# dt = cfl_time_step(0.4) capped at t_end - t and Manning friction (dry_tol
# 1e-6) after each step, to t = 20 s (at most 5000 steps). The observable is
# the depth-weighted centroid of the middle row, sum x h / sum h with
# x = (j + 0.5) dx, summed in column order.
M1_ROWS, M1_COLS, M1_T_END, M1_N_TRUE, M1_N_INIT, M1_ITERS = 3, 60, 20.0, 0.040, 0.080, 12


def m1_state():
    h = np.where(np.arange(M1_COLS)[None, :] < M1_COLS // 2, 1.0, 0.1) * np.ones((M1_ROWS, 1))
    z = np.zeros((M1_ROWS, M1_COLS))
    return z, h, np.zeros_like(h), np.zeros_like(h)


def m1_centroid(h_row, dh_row):
    """(value, derivative) of sum x h / sum h with the Dual division rule."""
    num = den = dnum = dden = 0.0
    for j in range(M1_COLS):
        x = (j + 0.5) * 1.0
        num += h_row[j] * x
        dnum += dh_row[j] * x
        den += h_row[j]
        dden += dh_row[j]
    return num / den, (dnum * den - num * dden) / (den * den)


def m1_newton(centroid_and_derivative):
    """The demo's Newton iteration (m1_inverse_manning_demo.rs:124-146) given
    n -> (centroid, d centroid / dn); returns rows (iter, n, centroid, loss,
    dc_dn, step) and the target centroid."""
    c_target = centroid_and_derivative(M1_N_TRUE)[0]
    n = M1_N_INIT
    rows = []
    for it in range(M1_ITERS):
        c, dc = centroid_and_derivative(n)
        err = c - c_target
        step = -err / dc if abs(dc) > 1e-12 else 0.0
        rows.append((it, n, c, err * err, dc, step))
        n = min(max(n + step, 1e-4), 1.0)
    return np.array(rows), c_target


def assert_matches_m1_record(rows, table, dc=0.0):
    """Rows against the reference's CSV (n and centroid to 10 decimals, the
    rest to 10 significant digits). `dc` is the absolute centroid difference
    allowed between the two runs (0 when both use the same pow; a correctly
    rounded pow moves the centroid by ~1e-14): near convergence the loss
    err^2 and the step -err / dc_dn inherit it through err = c - c_target."""
    assert rows.shape == table.shape
    for got, ref in zip(rows, table):
        it = int(ref[0])
        assert abs(got[1] - ref[1]) <= 6e-11, (it, "n", got[1], ref[1])
        assert abs(got[2] - ref[2]) <= 6e-11, (it, "centroid", got[2], ref[2])
        err_tol = {3: 2.0 * np.sqrt(ref[3]) * dc + dc * dc, 4: 0.0, 5: dc / abs(ref[4])}
        for k, name in ((3, "loss"), (4, "dc_dn"), (5, "step")):
            tol = 6e-10 * abs(ref[k]) + err_tol[k] + 1e-22
            assert abs(got[k] - ref[k]) <= tol, (it, name, got[k], ref[k])
