"""Builds ``libclayfluid.so`` (the C-ABI library) in-tree with nvcc for sm_100a.

``python -m clay_engine_b200.build`` or ``clay_engine_b200.build.build()``. Translation
units that must round exactly as written (the bake, the cell build, the reference-mode
neighbour passes, the host object model) are compiled with ``-fmad=false``; the fast-mode
neighbour passes with ``-fmad=true``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libclayfluid.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr"]
UNITS = [("kern_ref.cu", ["-fmad=false"]), ("kern_fast.cu", ["-fmad=true"]),
         ("clay_api.cu", ["-fmad=false"]), ("splat_static.cu", ["-fmad=false"]), ("clay_server.cu", [])]
HEADERS = ["clay_device.cuh", "launch.h"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libclayfluid.so")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, u) for u, _ in UNITS] + [os.path.join(CSRC, h) for h in HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "clay_fluid.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    nvcc = _nvcc()
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    for unit, flags in UNITS:
        obj = os.path.join(OUT_DIR, unit.replace(".cu", ".o"))
        cmd = [nvcc, *ARCH, *COMMON, *flags, "-c", os.path.join(CSRC, unit), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
