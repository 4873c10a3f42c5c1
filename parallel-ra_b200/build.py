"""Build recipe for the B200 engine (sm_100a) and its C++ API layer.

Outputs, in-tree next to this file:
  * libra_b200.so -- CUDA kernels + the C ABI of include/ra_engine.h
  * libparallel_ra.so -- the source-compatible C++ classes (relation, RAM,
    parallel_join, ..., LIE) over that C ABI
Run ``python parallel-ra_b200/build.py``; it is also what
``__graft_entry__.build()`` calls.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

ENGINE_SRCS = [os.path.join(HERE, "csrc", "ra_engine.cu")]   # includes csrc/ra_noalloc.cu
# every source of the engine's single translation unit (ra_engine.cu includes the rest)
ENGINE_DEPS = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [
    os.path.join(ROOT, "include", "ra_engine.h")]
ENGINE_LIB = os.path.join(HERE, "libra_b200.so")

CXX_DIR = os.path.join(HERE, "cxx")
CXX_SRCS = [os.path.join(CXX_DIR, "parallel_ra.cpp")]
CXX_LIB = os.path.join(HERE, "libparallel_ra.so")


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_engine(force=False):
    if force or _stale(ENGINE_LIB, ENGINE_DEPS):
        _run([NVCC, *ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
              "-I", os.path.join(ROOT, "include"), "-o", ENGINE_LIB, *ENGINE_SRCS])


def build_cxx(force=False):
    deps = CXX_SRCS + [os.path.join(CXX_DIR, "src", f) for f in os.listdir(os.path.join(CXX_DIR, "src"))] + [ENGINE_LIB]
    if os.path.exists(CXX_SRCS[0]) and (force or _stale(CXX_LIB, deps)):
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-I", os.path.join(ROOT, "include"),
              "-I", os.path.join(CXX_DIR, "src"), "-o", CXX_LIB, *CXX_SRCS, "-L", HERE, "-lra_b200",
              f"-Wl,-rpath,{HERE}", "-Wl,-rpath,$ORIGIN"])


# the parallel-RA checkout whose program sources are compiled against cxx/src
# (given by the caller; without it the binaries already in cxx/bin/ are used)
REFERENCE = os.environ.get("RA_REFERENCE", "")
BIN_DIR = os.path.join(CXX_DIR, "bin")


GENERATED_PROGRAMS = ["worstcase-110-terms-4-m"]


def build_reference_programs(force=False):
    """Compile the reference's own program sources, unchanged, against cxx/src.

    A reference program includes "../src/parallel_RA_inc.h".  The source is fed
    to g++ on stdin from cxx/tests/, so that include resolves to
    cxx/src/parallel_RA_inc.h; nothing is copied.  Only possible where the
    reference tree exists; the binaries in cxx/bin/ are used elsewhere.
    """
    if not REFERENCE:
        return
    progs = {"TC": os.path.join(REFERENCE, "tests", "transitive_closure.cpp")}
    for name in GENERATED_PROGRAMS:   # the reference's generated analyses (wide tuples)
        progs[name] = os.path.join(REFERENCE, "tests", name + ".cpp")
    os.makedirs(os.path.join(CXX_DIR, "tests"), exist_ok=True)
    os.makedirs(BIN_DIR, exist_ok=True)
    for name, src in progs.items():
        out = os.path.join(BIN_DIR, name)
        if not os.path.exists(src):
            continue
        if not (force or _stale(out, [src, CXX_LIB, os.path.join(CXX_DIR, "src", "parallel_RA_inc.h")])):
            continue
        cmd = ["g++", "-std=c++17", "-O2", "-x", "c++", "-", "-x", "none", "-o", out, "-L", HERE,
               "-lparallel_ra", "-lra_b200", f"-Wl,-rpath,{HERE}", "-Wl,-rpath,$ORIGIN/../.."]
        print(" ".join(cmd), "<", src, flush=True)
        with open(src, "rb") as f:
            subprocess.run(cmd, check=True, stdin=f, cwd=os.path.join(CXX_DIR, "tests"))


def build(force=False):
    build_engine(force)
    build_cxx(force)
    build_reference_programs(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
