"""Build recipe of libscb_b200.so (sm_100a) with nvcc, in-tree.

    python -m scbf_b200.build          # or __graft_entry__.build()

The shared library links the CUDA runtime statically, so it loads on hosts without a GPU
(entry points then return SCB_ERR_INTERNAL_STATE "no CUDA device available").
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libscb_b200.so")

SOURCES = ["scb_api.cu", "scb_kernels.cu", "scb_server.cu", "scb_fastx.cu", "scb_hostpack.cpp"]
HEADERS = ["scb_device.cuh", "scb_kernels.cuh", "scb_internal.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
         "-Xptxas", "-O3", "-cudart", "static"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "scb.h"), __file__]
    if not force and not _stale(LIB, deps):
        return LIB
    objs = []
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    for src in SOURCES:
        obj = os.path.join(bdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc(), *ARCH, *FLAGS, *(extra or []), "-I", os.path.join(ROOT, "include"), "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", *objs, "-o", tmp, "-lpthread", "-lz"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


WORKLOADS_SRC = os.path.join(CSRC, "scb_workloads.cpp")
WORKLOADS_LIB = os.path.join(HERE, "libscb_workloads.so")


def build_workloads(force: bool = False) -> str:
    """Host-only helper library of the seeded workload generators (g++)."""
    if not force and not _stale(WORKLOADS_LIB, [WORKLOADS_SRC, __file__]):
        return WORKLOADS_LIB
    tmp = WORKLOADS_LIB + ".tmp"
    subprocess.run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", WORKLOADS_SRC, "-o", tmp],
                   check=True)
    os.replace(tmp, WORKLOADS_LIB)
    return WORKLOADS_LIB


def build_all(force: bool = False, verbose: bool = False) -> None:
    build(force=force, verbose=verbose)
    build_workloads(force=force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
    build_workloads(force="--force" in sys.argv)
