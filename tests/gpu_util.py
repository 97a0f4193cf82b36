"""Helpers for the GPU parity tests (compare the CUDA path with the oracle)."""
from __future__ import annotations

import numpy as np

# Parity bar: max relative error <= 1e-10 in h/hu/hv (normwise: max |gpu-ref|
# over max |ref| of the field), and identical wet masks except for cells
# within 1e-12 of the dry threshold.
RTOL = 1e-10
H_DRY = 1e-6


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.max(np.abs(b)) if b.size else 0.0
    d = np.max(np.abs(a - b)) if a.size else 0.0
    if scale == 0.0:
        return d
    return d / scale


def parity_errors(gpu, ref):
    """Relative errors of (h, hu, hv): depth against max |h|; both momentum
    components against the momentum scale max(|hu|, |hv|) (a component that
    is identically zero in exact arithmetic, e.g. hv in uniform x-flow, only
    carries roundoff and has no scale of its own)."""
    h_s = float(np.max(np.abs(ref[0]))) if ref[0].size else 0.0
    q_s = max(float(np.max(np.abs(ref[1]))), float(np.max(np.abs(ref[2])))) if ref[1].size else 0.0
    out = []
    for a, b, s in zip(gpu, ref, (h_s, q_s, q_s)):
        d = float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if np.size(a) else 0.0
        out.append(d / s if s > 0.0 else d)
    return out


def assert_parity(gpu, ref, rtol=RTOL, what=""):
    names = ("h", "hu", "hv")
    for name, a, b in zip(names, gpu, ref):
        assert np.all(np.isfinite(a) == np.isfinite(b)), f"{what}{name}: finiteness differs"
    for name, e in zip(names, parity_errors(gpu, ref)):
        assert e <= rtol, f"{what}{name}: rel err {e:.3e} > {rtol:.1e}"
    hg, hr = np.asarray(gpu[0]), np.asarray(ref[0])
    mask_diff = (hg > H_DRY) != (hr > H_DRY)
    near = np.abs(hr - H_DRY) <= 1e-12
    assert not np.any(mask_diff & ~near), f"{what}wet mask differs at {np.argwhere(mask_diff & ~near)[:5]}"


def exact_fraction(gpu, ref):
    tot = 0
    same = 0
    for a, b in zip(gpu, ref):
        tot += a.size
        same += int(np.sum(a == b))
    return same / max(tot, 1)


def to_dev(*arrs):
    import torch
    return [torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda") for a in arrs]


def to_host(*ts):
    import torch
    torch.cuda.synchronize()
    return [t.detach().cpu().numpy() for t in ts]
