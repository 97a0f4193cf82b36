"""The hand-written reverse functions of the adjoint step (hydroflux_b200/csrc/
hf_adjoint_math.cuh) against the oracle's forward-mode Dual evaluation of the
same functions, on the CPU: for random inputs x, directions v and output
adjoints lam, lam . (J v) from the Dual tangents must equal v . (J^T lam) from
the reverse function. Covers the HLLC branches (wet/wet, dry-bed sides,
upwind and star states, the s* denominator guard, exact ties of the wave-speed
max/min), the hydrostatic reconstruction, Manning friction (with the Manning
derivative, dry and zero-momentum cells) and every ghost kind including the
Manning normal-depth dry-inflow ghost."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "native", "adjoint_math_check.cu")
OUT_DIR = os.path.join(HERE, "native", "_build")
OUT = os.path.join(OUT_DIR, "libadjoint_math_check.so")

_D = C.POINTER(C.c_double)


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    return None


@pytest.fixture(scope="module")
def chk():
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    deps = [SRC, os.path.join(ROOT, "hydroflux_b200", "csrc", "hf_adjoint_math.cuh"),
            os.path.join(ROOT, "hydroflux_b200", "csrc", "hf_device.cuh"),
            os.path.join(ROOT, "oracle", "hf_oracle.hpp")]
    if not os.path.exists(OUT) or any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in deps):
        os.makedirs(OUT_DIR, exist_ok=True)
        subprocess.run([nvcc, "-std=c++17", "-O1", "--fmad=false", "-Xcompiler", "-fPIC",
                        "-Xcompiler", "-ffp-contract=off", "-shared",
                        "-I", os.path.join(ROOT, "hydroflux_b200", "csrc"),
                        "-I", os.path.join(ROOT, "oracle"), "-I", os.path.join(ROOT, "include"),
                        SRC, "-o", OUT], check=True)
    lib = C.CDLL(OUT)
    lib.chk_hllc.argtypes = [_D, _D, _D, _D]
    lib.chk_wb.argtypes = [_D, C.c_double, _D, _D, _D]
    lib.chk_friction.argtypes = [_D, _D, C.c_double, C.c_double, _D, _D]
    lib.chk_ghost.argtypes = [C.c_int, C.c_int, C.c_double, _D, _D, _D, _D, _D, _D, _D]
    lib.chk_set_pow_mode.argtypes = [C.c_int]
    lib.chk_set_pow_mode(1)
    return lib


def p(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_D)


def call(fn, *arrays_and_scalars):
    keep, args = [], []
    for a in arrays_and_scalars:
        if isinstance(a, np.ndarray):
            arr, ptr = p(a)
            keep.append(arr)
            args.append(ptr)
        else:
            args.append(a)
    out, optr = p(np.zeros(3))
    fn(*args, optr)
    return out


def close(out, rtol=1e-12, lam=None, v=None):
    """Forward and reverse sides agree to rounding, measured against the sum
    of the absolute terms of the reverse side (cancellation scale), with an
    absolute floor of 1e-14 |lam|_1 |v|_1 for cancellation inside a term
    (e.g. (h + z) - z against h on films of 1e-13 m)."""
    fwd, rev, terms = out
    atol = 1e-14 * np.abs(lam).sum() * np.abs(v).sum() if lam is not None else 1e-300
    return abs(fwd - rev) <= rtol * max(terms, abs(fwd), abs(rev)) + atol


def depth(rng):
    kind = rng.integers(0, 6)
    if kind == 0:
        return 0.0
    if kind == 1:
        return float(rng.uniform(0, 1e-12))  # dry for HLLC
    if kind == 2:
        return float(rng.uniform(1e-12, 1e-5))  # wet, below the velocity cutoff
    return float(rng.uniform(1e-4, 5.0))


def state(rng, h, speed=3.0):
    """(h, h u_n, h u_t) with velocities of a few m/s."""
    return [h, h * rng.normal() * speed, h * rng.normal() * speed]


def test_hllc_reverse_is_transpose_of_dual(chk):
    rng = np.random.default_rng(1)
    seen = set()
    for _ in range(20000):
        hl, hr = depth(rng), depth(rng)
        x = np.array(state(rng, hl) + state(rng, hr))
        v, lam = rng.normal(size=6), rng.normal(size=3)
        out = call(chk.chk_hllc, x, v, lam)
        assert close(out, lam=lam, v=v), (x, v, lam, out)
        seen.add((hl > 1e-12, hr > 1e-12))
    assert seen == {(True, True), (True, False), (False, True), (False, False)}


def test_hllc_extreme_velocities(chk):
    """Films of ~1e-6 m carrying ~1e3 m/s: derivatives like qn / h^2 reach
    1e8 and cancel, so both sides agree only to ~1e-9 of the terms."""
    rng = np.random.default_rng(5)
    for _ in range(5000):
        hl, hr = depth(rng), depth(rng)
        x = np.array([hl, rng.normal() * max(hl, 1e-3) * 3, rng.normal() * max(hl, 1e-3),
                      hr, rng.normal() * max(hr, 1e-3) * 3, rng.normal() * max(hr, 1e-3)])
        v, lam = rng.normal(size=6), rng.normal(size=3)
        out = call(chk.chk_hllc, x, v, lam)
        assert close(out, 1e-8, lam=lam, v=v), (x, v, lam, out)


def test_hllc_ties_and_guard(chk):
    # symmetric states: un_l - cl == un_r - cr ties in the min / max
    for x in ([1.0, 0.0, 0.3, 1.0, 0.0, -0.2], [2.0, 1.0, 0.0, 2.0, 1.0, 0.5],
              [1.0, 0.5, 0.0, 1.0, -0.5, 0.0], [1e-3, 0.0, 0.0, 1e-3, 0.0, 0.0]):
        x = np.array(x)
        rng = np.random.default_rng(2)
        for _ in range(50):
            v, lam = rng.normal(size=6), rng.normal(size=3)
            out = call(chk.chk_hllc, x, v, lam)
            assert close(out, lam=lam, v=v), (x, out)


def test_wb_face_reverse_is_transpose_of_dual(chk):
    rng = np.random.default_rng(3)
    for _ in range(20000):
        hl, hr = depth(rng), depth(rng)
        zf = float(rng.choice([0.0, rng.uniform(-5, 5)]))
        x = np.array(state(rng, hl) + state(rng, hr))
        v, lam = rng.normal(size=6), rng.normal(size=4)
        out = call(chk.chk_wb, x, zf, v, lam)
        assert close(out, lam=lam, v=v), (x, zf, v, lam, out)


def test_friction_reverse_is_transpose_of_dual(chk):
    rng = np.random.default_rng(4)
    for k in range(5000):
        h = float(rng.choice([0.0, 5e-7, rng.uniform(1e-6, 1e-3), rng.uniform(0.01, 4.0)]))
        hu, hv = (0.0, 0.0) if k % 7 == 0 else tuple(rng.normal(size=2) * 3.0 * h)
        n = 0.0 if k % 11 == 0 else float(rng.uniform(0.01, 0.1))
        x = np.array([h, hu, hv, n])
        v, lam = rng.normal(size=4), rng.normal(size=3)
        dt = float(rng.uniform(0.01, 5.0))
        out = call(chk.chk_friction, x, v, dt, 1e-6, lam)
        assert close(out, lam=lam, v=v), (x, v, lam, dt, out)


@pytest.mark.parametrize("side", [0, 1, 2, 3])
@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_ghost_reverse_is_transpose_of_dual(chk, side, kind):
    rng = np.random.default_rng(10 + 4 * side + kind)
    for k in range(300):
        z = rng.uniform(0, 2, size=9) if k % 3 else np.linspace(0, 0.5, 9)
        n = rng.uniform(0.02, 0.08, size=9)
        vn = rng.normal(size=9)
        h = 0.0 if k % 2 == 0 else float(rng.uniform(0.01, 2.0))  # dry cells take the inflow ghost
        x = np.array([h, rng.normal(), rng.normal()])
        v, lam = rng.normal(size=3), rng.normal(size=3)
        value = float(rng.uniform(-30, 30)) if kind == 2 else float(rng.uniform(0.1, 3.0))
        out = call(chk.chk_ghost, side, kind, value, z, n, vn, x, v, lam)
        assert close(out, lam=lam, v=v), (side, kind, x, out)
