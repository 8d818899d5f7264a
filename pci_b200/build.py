"""Build libpci_gpu.so in-tree with nvcc for sm_100a.

The library is plain CUDA C++ behind the C ABI of include/pci_gpu.h; it does
not link against libtorch or Python.  Objects go to pci_b200/_build/, the
shared library to pci_b200/lib/libpci_gpu.so.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libpci_gpu.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                 "--expt-relaxed-constexpr"]
# Per-unit extra flags.  The H-build keeps the reference's operation order with
# separately rounded multiplies and adds (no fused multiply-add contraction).
UNITS = {
    "hbuild.cu": ["-fmad=false"],
    "spmm.cu": [],
    "davidson.cu": [],
    "pci_gpu.cu": [],
}
HEADERS = ["pci_internal.h", os.path.join("..", "..", "include", "pci_gpu.h")]


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def build(verbose: bool = False, force: bool = False, extra: list | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdr_t = max(_mtime(os.path.join(SRC, hh)) for hh in HEADERS)
    objs = []
    for unit, flags in UNITS.items():
        src = os.path.join(SRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _mtime(obj) < max(_mtime(src), hdr_t):
            cmd = [NVCC] + COMMON + flags + (extra or []) + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
    if force or _mtime(LIB) < max(_mtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-lcusolver", "-lcublas", "-Xlinker", f"-rpath,{CUDA_HOME}/lib64"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
    print(LIB)
