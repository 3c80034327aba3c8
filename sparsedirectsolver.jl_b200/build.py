"""Build the native libraries of the package in-tree.

* ``libsdsb200.so``: the numeric phase, CUDA for sm_100a (nvcc), C ABI of
  ``include/sdsb200.h``;
* ``libsdsb200_analysis.so``: the host analysis (g++), C ABI of
  ``include/sdsb200_analysis.h``.

Run ``python sparsedirectsolver.jl_b200/build.py`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

NUMERIC_SOURCES = [
    "numeric/plan.cu",
    "numeric/factor_kernels.cu",
    "numeric/dense_kernels.cu",
    "numeric/pivot_kernels.cu",
    "numeric/solve_kernels.cu",
    "numeric/solve_dataflow.cu",
    "numeric/pinv_kernels.cu",
    "numeric/schur_kernels.cu",
    "numeric/adjoint_kernels.cu",
    "numeric/tc_kernels.cu",
    "numeric/capi.cu",
]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_analysis(force: bool = False) -> str:
    out = os.path.join(HERE, "libsdsb200_analysis.so")
    src = os.path.join(CSRC, "analysis", "analysis.cpp")
    hdr = os.path.join(INCLUDE, "sdsb200_analysis.h")
    if force or _newer(out, [src, hdr]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-o", out, src])
    return out


# Units that restate the reference's scalar in-front arithmetic: no fused multiply-add, so that their
# values, and the pivots and inertia that depend on exact cancellation, match the reference's
NO_CONTRACTION = {"factor_kernels.cu", "pivot_kernels.cu"}


def build_numeric(force: bool = False) -> str:
    out = os.path.join(HERE, "libsdsb200.so")
    srcs = [os.path.join(CSRC, s) for s in NUMERIC_SOURCES]
    deps = srcs + [os.path.join(CSRC, "numeric", h) for h in os.listdir(os.path.join(CSRC, "numeric"))
                   if h.endswith((".cuh", ".h"))] + [os.path.join(INCLUDE, "sdsb200.h")]
    if not (force or _newer(out, deps)):
        return out
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s).replace(".cu", ".o"))
        fmad = ["--fmad=false"] if os.path.basename(s) in NO_CONTRACTION else []
        _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE,
              "--expt-relaxed-constexpr", *fmad, "-c", s, "-o", o])
        objs.append(o)
    _run([NVCC, *ARCH, "-shared", "-o", out, *objs, "-lcudart"])
    return out


def build(force: bool = False) -> None:
    build_analysis(force)
    build_numeric(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
