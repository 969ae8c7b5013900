"""Build ``libgralprog.so`` (the C-ABI solver library) in-tree with nvcc for sm_100a.

Floating point: ``--fmad=false`` keeps every multiply and add separately rounded (the reference's
.NET JIT does not contract them), division and square root stay IEEE-rounded (no fast-math), and
the host-side set-up is compiled with ``-ffp-contract=off`` for the same reason.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgralprog.so")
SOURCES = ["prog_host.cu", "prog_gs.cu", "prog_kernels.cu", "prog_gff.cu", "prog_prep.cu", "prog_wind.cu", "prog_runner.cu", "prog_noalloc.cu", "prog_adjoint.cu"]
HEADERS = ["prog_common.cuh", "prog_ctx.cuh", "prog_kernels.cuh", "prog_level.cuh", "prog_gff.cuh", "prog_prep.cuh", "adj_level.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libgralprog.so")


def flags(extra=()):
    return (ARCH + ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler",
                    "-fPIC,-ffp-contract=off,-fno-fast-math", "-I", os.path.join(ROOT, "include"),
                    "-I", CSRC] + list(extra))


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "gral_prog.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not stale():
        return LIB
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    nv = nvcc()
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nv] + flags(extra) + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nv] + ARCH + ["-shared", "-o", tmp] + objs
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
