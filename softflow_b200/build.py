"""Builds libsoftflow_b200.so in-tree with nvcc for sm_100a.

Usage: python -m softflow_b200.build  (or softflow_b200.build.build()).

Translation units and their floating-point contract:
  lattice_f64.cu, markers.cu  --fmad=false: FP64 paths keep the reference's
                              rounding (no fused multiply-add contraction);
  lattice_f32.cu, scan.cu, context.cu: default contraction;
  host_setup.cpp (g++)        -ffp-contract=off.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsoftflow_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

UNITS = [
    ("lattice_f64.cu", ["--fmad=false"]),
    ("lattice_f32.cu", []),
    ("markers.cu", ["--fmad=false"]),
    ("spread_standalone.cu", ["--fmad=false"]),
    ("spread_noalloc.cu", []),
    ("scan.cu", []),
    ("mlp.cu", []),
    ("learned_step.cu", ["--fmad=false"]),
    ("chemistry.cu", ["--fmad=false"]),
    ("context.cu", []),
]
HOST_UNITS = [("host_setup.cpp", ["-ffp-contract=off"]), ("host_io.cpp", ["-ffp-contract=off"])]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "softflow_gpu.h"))
    objs = []
    nvcc = _nvcc()
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers + [__file__]):
            cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", "-c", s, "-o", o, *extra]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    for src, extra in HOST_UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers + [__file__]):
            cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-c", s, "-o", o, *extra]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-ldl",
               "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
