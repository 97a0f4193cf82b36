"""The kernels' division helpers (hydroflux_b200/csrc/hf_arith.h) are
bit-identical to IEEE division on the GPU: the reciprocal division by a grid
spacing (Markstein's correction), the zero-safe division and the
positive-divisor variant, on 1.6 * 10^9 counter-based random pairs per
helper covering typical, random and wide-range divisors, the edges of the
reciprocal path's exponent window, zeros, subnormals and infinities."""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "division_check.cu")
OUT = os.path.join(HERE, "native", "_build", "division_check")


def test_division_helpers_match_ieee():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", SRC, "-o", OUT],
                   check=True)
    r = subprocess.run([OUT, str(1 << 28)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("mismatches div_recip 0, div_rn_pos 0, div_rn 0") == 6
