"""Build of the in-tree CUDA library `libivp.so` (sm_100a).

`python -m implicitvelocityprojection_b200.build` compiles
`csrc/ivp_engine.cu` with nvcc for `compute_100a`/`sm_100a` into
`implicitvelocityprojection_b200/libivp.so`.  The library exports the C ABI
declared in `include/ivp.h` and links only the CUDA runtime.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libivp.so")
SOURCES = ["ivp_engine.cu", "ivp_noalloc.cu"]
DEPS = ["ivp_engine.cu", "ivp_noalloc.cu", "ivp_kernels.cuh", "ivp_device.cuh", "ivp_scan.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the IVP engine needs the CUDA toolkit to build")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    paths = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(REPO, "include", "ivp.h")]
    return any(os.path.getmtime(p) > t for p in paths)


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and not _stale():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + list(extra or []) + ["-I", os.path.join(REPO, "include"), "-o", LIB + ".tmp"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose and (res.stdout or res.stderr):
        print(res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
    print("built", LIB)
