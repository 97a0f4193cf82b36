"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/hf_oracle_capi.cpp into oracle/libhf_oracle.so with the
flags that keep its rounding identical to the Rust reference's: no FMA
contraction, no fast-math. OpenMP only splits independent per-cell passes
(like the reference's optional rayon row chunks), so results do not depend
on the thread count.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "hf_oracle_capi.cpp")
HDRS = [os.path.join(HERE, "hf_oracle.hpp"),
        os.path.join(HERE, "..", "include", "hydroflux_gpu.h"),
        os.path.join(HERE, "..", "hydroflux_b200", "csrc", "hf_pow.h")]
OUT = os.path.join(HERE, "libhf_oracle.so")

CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
            "-fno-fast-math", "-fopenmp", "-Wall", "-Wno-unused-function"]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t_out = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t_out for p in [SRC, *HDRS])


def build(force: bool = False) -> str:
    if force or needs_build():
        cmd = ["g++", *CXXFLAGS, SRC, "-o", OUT + ".tmp"]
        subprocess.run(cmd, check=True)
        os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
