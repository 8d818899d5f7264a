"""Build libpci_gpu.so in-tree with nvcc for sm_100a.

The library is plain CUDA C++ behind the C ABI of include/pci_gpu.h; it does
not link against libtorch or Python.  Objects go to pci_b200/_build/, the
shared library to pci_b200/lib/libpci_gpu.so.  Translation units compile in
parallel; the Hamiltonian-build kernels are instantiated once per electron
count (hbuild_ne.cu with -DPCI_NE=1..8).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

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
# The Hamiltonian build keeps the reference's operation order with separately
# rounded multiplies and adds (no fused multiply-add contraction).
NOFMA = ["-fmad=false"]
NE_MAX = 8

# (object name, source, extra flags)
UNITS = [("hbuild", "hbuild.cu", NOFMA)] + \
    [(f"hbuild_ne{n}", "hbuild_ne.cu", NOFMA + [f"-DPCI_NE={n}"]) for n in range(1, NE_MAX + 1)] + \
    [("spmm", "spmm.cu", []), ("davidson", "davidson.cu", []), ("pci_gpu", "pci_gpu.cu", []),
     ("noalloc", "noalloc.cu", []), ("pci_io", "pci_io.cpp", []), ("mlp", "mlp.cu", []), ("lsj", "lsj.cu", NOFMA), ("csf", "csf.cu", []), ("pt", "pt.cu", []),
     ("batch", "batch.cu", [])]
HEADERS = ["pci_internal.h", "hbuild_impl.cuh", "mlp_tc.cuh", os.path.join("..", "..", "include", "pci_gpu.h"),
           os.path.join("..", "..", "include", "pci_io.h"), os.path.join("..", "..", "include", "pci_batch.h")]


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def build(verbose: bool = False, force: bool = False, extra: list | None = None, jobs: int = 0) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdr_t = max(_mtime(os.path.join(SRC, hh)) for hh in HEADERS)
    todo, objs = [], []
    for name, unit, flags in UNITS:
        src = os.path.join(SRC, unit)
        obj = os.path.join(BUILD, name + ".o")
        objs.append(obj)
        if force or _mtime(obj) < max(_mtime(src), hdr_t):
            todo.append([NVCC] + COMMON + flags + (extra or []) + ["-c", src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)

    if todo:
        with ThreadPoolExecutor(max_workers=jobs or max(1, os.cpu_count() or 1)) as ex:
            for f in [ex.submit(run, c) for c in todo]:
                f.result()
    if force or _mtime(LIB) < max(_mtime(o) for o in objs):
        run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xlinker", f"-rpath,{CUDA_HOME}/lib64"])
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
    print(LIB)
