"""In-tree build of the CUDA library lbm_b200/liblbm_b200.so for sm_100a.

    python -m lbm_b200.build          # or lbm_b200.build.build()

Each .cu/.cpp under lbm_b200/csrc is compiled by nvcc into an object (the
FP64 kernels with -fmad=false so their arithmetic keeps the reference's
rounding), then linked into one shared library with the CUDA runtime linked
statically.  Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblbm_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "-I" + os.path.join(ROOT, "include")]
# Per-file extra flags.  The FP64 kernels must not contract a*b+c into FMA.
EXTRA = {
    "kernels_fp64.cu": ["-fmad=false"],
}


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    hdr_time = _newest(headers)
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp"))):
        name = os.path.basename(src)
        if name.startswith("main_"):
            continue  # command-line front ends are linked separately
        obj = os.path.join(OBJ, name + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time):
            continue
        cmd = [nvcc()] + ARCH + COMMON + EXTRA.get(name, []) + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [nvcc(), "-x", "cu"] + cmd[1:]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
