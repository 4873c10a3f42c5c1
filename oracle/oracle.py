"""ctypes binding of the CPU oracle (oracle/libra_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker.  It exposes the same builder
methods as the product's Python binding (relation / load_rows / scc /
add_relation / join / copy / depend / execute / history / dump_full), so one
program definition drives both.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libra_oracle.so")

DELTA, FULL = 0, 1
COPY, ACOPY, COPY_FILTER = 0, 1, 2

_lib = None


def reference_root() -> str | None:
    """The parallel-RA checkout oracle/Makefile builds from ($RA_REFERENCE or its
    default), or None when that tree is not on this machine."""
    r = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True)
    path = r.stdout.strip()
    return path if r.returncode == 0 and os.path.isdir(os.path.join(path, "src")) else None


def build() -> None:
    """Compile the restatement (and, when the reference tree exists, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if reference_root():
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"-j{os.cpu_count() or 4}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        u64p = C.POINTER(C.c_uint64)
        i32p = C.POINTER(C.c_int)
        L.oracle_create.restype = P
        L.oracle_destroy.argtypes = [P]
        L.oracle_relation.argtypes = [P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_char_p, C.c_int]
        L.oracle_load_rows.argtypes = [P, C.c_int, u64p, C.c_uint64]
        L.oracle_scc.argtypes = [P, C.c_int, C.c_int]
        L.oracle_scc_add_relation.argtypes = [P, C.c_int, C.c_int, C.c_int]
        L.oracle_scc_add_join.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, i32p, C.c_int]
        L.oracle_scc_add_copy.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, i32p, C.c_int, C.c_int]
        L.oracle_depend.argtypes = [P, C.c_int, C.c_int]
        L.oracle_execute.argtypes = [P, C.c_int]
        L.oracle_history_len.argtypes = [P]
        L.oracle_history_len.restype = C.c_uint64
        L.oracle_history.argtypes = [P, u64p, C.c_uint64]
        L.oracle_history.restype = C.c_uint64
        L.oracle_full_count.argtypes = [P, C.c_int]
        L.oracle_full_count.restype = C.c_uint64
        L.oracle_dump_full.argtypes = [P, C.c_int, u64p, C.c_uint64]
        L.oracle_dump_full.restype = C.c_uint64
        L.oracle_fixpoint_seconds.argtypes = [P]
        L.oracle_fixpoint_seconds.restype = C.c_double
        L.oracle_tc_distance_histogram.argtypes = [u64p, u64p, C.c_uint64, C.c_uint64, u64p, C.c_uint64, C.c_int]
        L.oracle_tc_distance_histogram.restype = C.c_uint64
        _lib = L
    return _lib


def _u64(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _i32(seq):
    arr = (C.c_int * len(seq))(*seq)
    return arr


class OracleProgram:
    """Program builder over the CPU oracle."""

    def __init__(self):
        self._L = lib()
        self._p = self._L.oracle_create()
        self._arity = {}

    def close(self):
        if self._p:
            self._L.oracle_destroy(self._p)
            self._p = None

    def __del__(self):
        self.close()

    def relation(self, jcc, arity, tag, name, version=FULL):
        r = self._L.oracle_relation(self._p, jcc, arity, tag, name.encode(), version)
        if r < 0:
            raise ValueError("oracle: unsupported relation shape")
        self._arity[r] = arity
        return r

    def load_rows(self, rel, rows: np.ndarray):
        rows = np.ascontiguousarray(rows, dtype=np.uint64)
        self._L.oracle_load_rows(self._p, rel, _u64(rows), rows.shape[0])

    def scc(self, fixpoint, scc_id):
        return self._L.oracle_scc(self._p, int(bool(fixpoint)), scc_id)

    def add_relation(self, scc, rel, init_status):
        self._L.oracle_scc_add_relation(self._p, scc, rel, int(bool(init_status)))

    def join(self, scc, out, in0, ver0, in1, ver1, proj):
        self._L.oracle_scc_add_join(self._p, scc, out, in0, ver0, in1, ver1, _i32(proj), len(proj))

    def copy(self, scc, out, src, ver, proj, kind=COPY, pred=0):
        self._L.oracle_scc_add_copy(self._p, scc, kind, out, src, ver, _i32(proj), len(proj), pred)

    def depend(self, src_scc, dst_scc):
        self._L.oracle_depend(self._p, src_scc, dst_scc)

    def execute(self, batch_size=1):
        if self._L.oracle_execute(self._p, batch_size) != 0:
            raise RuntimeError("oracle execute failed")

    def history(self):
        """[(scc_id, [(sum_delta, sum_full), ...]), ...] in execution order."""
        n = self._L.oracle_history_len(self._p)
        buf = np.zeros(max(int(n), 1), dtype=np.uint64)
        self._L.oracle_history(self._p, _u64(buf), n)
        out, i = [], 0
        while i < n:
            sid, k = int(buf[i]), int(buf[i + 1])
            pairs = [(int(buf[i + 2 + 2 * j]), int(buf[i + 3 + 2 * j])) for j in range(k)]
            out.append((sid, pairs))
            i += 2 + 2 * k
        return out

    def full_count(self, rel):
        return int(self._L.oracle_full_count(self._p, rel))

    def dump_full(self, rel):
        """Full relation rows (data columns + id), lexicographically sorted."""
        n = self.full_count(rel)
        w = self._arity[rel] + 1
        buf = np.zeros((max(n, 1), w), dtype=np.uint64)
        got = self._L.oracle_dump_full(self._p, rel, _u64(buf), n)
        return buf[:got]

    def fixpoint_seconds(self):
        return float(self._L.oracle_fixpoint_seconds(self._p))


def tc_distance_histogram(edges: np.ndarray, n: int, cap: int = 4096, threads: int = 0) -> np.ndarray:
    """hist[d] = pairs (x, z) of the graph whose shortest path from x to z has d
    edges (the shortest cycle through x for z == x), over every source x.

    Independent of the reference's algorithm: semi-naive transitive closure adds
    the pairs at distance k + 2 in its k-th join iteration, so its per-iteration
    delta sizes must equal hist[2:], and its base (T = G) must hold hist[1] pairs.
    """
    src = np.ascontiguousarray(edges[:, 0], dtype=np.uint64)
    dst = np.ascontiguousarray(edges[:, 1], dtype=np.uint64)
    hist = np.zeros(cap, dtype=np.uint64)
    deep = lib().oracle_tc_distance_histogram(_u64(src), _u64(dst), src.size, n, _u64(hist), cap,
                                              threads or (os.cpu_count() or 1))
    if deep == 2 ** 64 - 1:
        raise ValueError("a shortest path is longer than the histogram holds")
    return hist[:deep + 1]

