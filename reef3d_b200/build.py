"""Builds libreef3d_b200.so in-tree for sm_100a with nvcc (no JIT cache).

The FP64 kernels are compiled with -fmad=false so products and sums round
separately, the way the reference's CPU build without FMA contraction does;
host code that builds the grid metrics is compiled with -ffp-contract=off
for the same reason.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libreef3d_b200.so")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
CUDA_INC = os.path.join(CUDA_HOME, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
               "-I" + CSRC, "-I" + INCLUDE] + ARCH

# (source, extra flags)
UNITS = [
    ("kernels_f64.cu", ["-fmad=false"]),
    ("kernels_f32.cu", ["-fmad=true"]),
    ("kernels_f32_tile.cu", ["-fmad=true"]),
    ("kernels_batch.cu", ["-fmad=true"]),
    ("noalloc.cu", ["-fmad=false"]),
    ("kernels_common.cu", ["-fmad=false"]),
    ("grid_metrics.cpp", []),
    ("api.cpp", []),
    ("batch.cpp", []),
    ("serve.cpp", []),
    ("state.cpp", []),
]
HEADERS = ["r3d_internal.h", "stencil_f64.cuh", "stencil_f32.cuh", "tile_host.h", "cell_f32.cuh", "handle.h", "batch_internal.h"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def _compile(unit, flags, verbose):
    src = os.path.join(CSRC, unit)
    obj = os.path.join(BUILD, unit + ".o")
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "reef3d_b200.h")]
    if _mtime(obj) >= max(_mtime(d) for d in deps):
        return obj
    cmd = [nvcc(), "-c", src, "-o", obj] + NVCC_COMMON + flags
    if unit.endswith(".cpp"):
        cmd = [os.environ.get("CXX", "g++"), "-c", src, "-o", obj, "-O2", "-std=c++17", "-fPIC",
               "-ffp-contract=off", "-Wall", "-I" + CSRC, "-I" + INCLUDE, "-I" + CUDA_INC]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return obj


def build(verbose=False, force=False):
    """Compile every unit (in parallel) and link the shared library."""
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda u: _compile(u[0], u[1], verbose), UNITS))
    if _mtime(LIB) < max(_mtime(o) for o in objs):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-Xlinker", "--no-undefined"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
