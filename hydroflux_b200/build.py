"""Build the sm_100a shared library hydroflux_b200/libhydroflux_gpu.so.

nvcc cross-compiles without a GPU. Floating-point flags keep the kernels'
rounding identical to the reference's Rust f64 code: no FMA contraction,
IEEE-rounded division and square root.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "libhydroflux_gpu.so")

SOURCES = ["hf_kernels.cu", "hf_tiles.cu", "hf_api.cu", "hf_noalloc.cu", "hf_batch.cu",
           "hf_serve.cu", "hf_adjoint.cu", "hf_calib.cu", "hf_io.cu"]
# hf_tiles.cu is compiled once more for the 32 x 32 tile geometry (the
# default macros give the 32 x 8 one; see hf_internal.h).
GEOM_LARGE = ("hf_tiles.cu", "hf_tiles_g32.o",
              ["-DHF_GEOM=g32", "-DHF_GEOM_INDEX=1", "-DHF_TILE_Y=32", "-DHF_THREADS=1024",
               "-DHF_MIN_BLOCKS=1"])
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true",
              "-prec-sqrt=true", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(INCLUDE, "hydroflux_gpu.h"))
    files.append(os.path.abspath(__file__))
    return files


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(f) > t for f in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not (force or needs_build()):
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    units = [(src, src.replace(".cu", ".o"), []) for src in SOURCES] + [GEOM_LARGE]
    objs, procs = [], []
    for src, name, defs in units:  # the translation units compile in parallel
        obj = os.path.join(objdir, name)
        cmd = [nvcc(), *GENCODE, *NVCC_FLAGS, *defs, "-I", INCLUDE, "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    tmp = OUT + ".tmp"
    subprocess.run([nvcc(), *GENCODE, "-shared", "-cudart", "static", "-o", tmp, *objs, "-lz"],
                   check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
