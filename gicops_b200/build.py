"""Builds libgicops_b200.so in-tree (gicops_b200/_lib/) for sm_100a with nvcc.

    python -m gicops_b200.build [--force]

The library holds the CUDA kernels, the C ABI declared in include/gicops_b200.h
and the host index builder.  Host C++ is compiled by /usr/bin/g++ (it carries
OpenMP); device code is compiled with -fmad=false so FP64 steps are not fused.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT, "libgicops_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off", "-ccbin", HOSTCXX, "-I" + os.path.join(ROOT, "include")]
# extra nvcc flags, e.g. GX_NVCC_FLAGS="-DGX_PEND=192" (recorded next to the library, so
# that a change of flags rebuilds it)
EXTRA = os.environ.get("GX_NVCC_FLAGS", "").split()
STAMP = os.path.join(OUT, "nvcc_flags.txt")
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include")]


def sources():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")) + glob.glob(os.path.join(SRC, "*.cpp")))


def _deps():
    return sources() + glob.glob(os.path.join(SRC, "*.h")) + glob.glob(os.path.join(SRC, "*.cuh")) + \
        [os.path.join(ROOT, "include", "gicops_b200.h"), __file__]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    if (open(STAMP).read() if os.path.exists(STAMP) else "") != " ".join(EXTRA):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(OUT, "obj", os.path.basename(src) + ".o")
        if src.endswith(".cu"):
            cmd = [NVCC, *ARCH, *CUFLAGS, *EXTRA, "-c", src, "-o", obj]
        else:
            cmd = [HOSTCXX, *CXXFLAGS, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-ccbin", HOSTCXX, "-Xcompiler", "-fopenmp", "-o", tmp, *objs,
           "-lcudart", "-lgomp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    shutil.move(tmp, LIB)
    with open(STAMP, "w") as f:
        f.write(" ".join(EXTRA))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
