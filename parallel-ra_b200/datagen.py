"""Seeded synthetic relations in parallel-RA's binary relation format.

Format (utility/tsv_to_bin.cpp:38-64, read by src/IO/parallel_io.cpp:115-213):
``<path>`` holds rows of ``arity + 1`` little-endian u64 -- the data columns
followed by an id column (tsv_to_bin writes the row index) -- and
``<path>.size`` holds ``"<rows>\\n<cols>"``.

Graphs:
  * ``erdos_renyi(n, m, seed)``: ``m`` distinct directed pairs ``(u, v)``,
    ``u != v``, endpoints uniform in ``[0, n)``, kept in first-draw order.
  * ``random_tree(n, seed)``: rooted tree built breadth-first; every node taken
    off the queue gets ``U{1..4}`` children until ``n`` nodes exist; edges are
    ``(parent, child)``.
  * ``batched_instances(count, seed)``: per-instance ER graphs with ``n``
    log-uniform in ``[64, 16384]`` and mean out-degree uniform in ``[0.8, 2.0]``.
"""
from __future__ import annotations

import math
import os

import numpy as np


def erdos_renyi(n: int, m: int, seed: int) -> np.ndarray:
    """``m`` distinct directed edges without self-loops, shape ``(m, 2)`` u64."""
    if m > n * (n - 1):
        raise ValueError("more edges than ordered pairs")
    rng = np.random.Generator(np.random.PCG64(seed))
    keys = np.empty(0, dtype=np.uint64)
    order = np.empty(0, dtype=np.int64)
    drawn = 0
    while keys.size < m:
        want = int((m - keys.size) * 1.1) + 64
        u = rng.integers(0, n, size=want, dtype=np.uint64)
        v = rng.integers(0, n, size=want, dtype=np.uint64)
        ok = u != v
        k = u[ok] * np.uint64(n) + v[ok]
        allk = np.concatenate([keys, k])
        allo = np.concatenate([order, drawn + np.arange(k.size, dtype=np.int64)])
        drawn += k.size
        uniq, first = np.unique(allk, return_index=True)
        sel = np.sort(first)
        keys = allk[sel]
        order = allo[sel]
    keys = keys[:m]
    return np.stack([keys // np.uint64(n), keys % np.uint64(n)], axis=1).astype(np.uint64)


def random_tree(n: int, seed: int) -> np.ndarray:
    """Breadth-first random tree, children per expanded node uniform in {1..4}."""
    rng = np.random.Generator(np.random.PCG64(seed))
    parents = np.empty(max(n - 1, 0), dtype=np.uint64)
    nxt = 1
    head = 0
    while nxt < n:
        k = int(rng.integers(1, 5))
        k = min(k, n - nxt)
        parents[nxt - 1: nxt - 1 + k] = head
        nxt += k
        head += 1
    child = np.arange(1, n, dtype=np.uint64)
    return np.stack([parents, child], axis=1)


def batched_sizes(count: int, seed: int) -> list[tuple[int, int, int]]:
    """(n, m, seed) per instance: n log-uniform in [64, 16384], degree U[0.8, 2.0]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(64), math.log(16384)))))
        deg = float(rng.uniform(0.8, 2.0))
        m = int(round(deg * n))
        out.append((n, m, seed * 1_000_003 + i))
    return out


def with_row_ids(pairs: np.ndarray) -> np.ndarray:
    """Append the tsv_to_bin id column (the row index) -> shape (rows, 3)."""
    rows = np.empty((pairs.shape[0], pairs.shape[1] + 1), dtype=np.uint64)
    rows[:, :-1] = pairs
    rows[:, -1] = np.arange(pairs.shape[0], dtype=np.uint64)
    return rows


def write_relation(path: str, rows: np.ndarray) -> None:
    """Write rows (data columns + id column) and the ``.size`` metadata file."""
    rows = np.ascontiguousarray(rows, dtype="<u8")
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "wb") as f:
        f.write(rows.tobytes())
    with open(path + ".size", "w") as f:
        f.write(f"{rows.shape[0]}\n{rows.shape[1] if rows.ndim == 2 else 3}")


def read_relation(path: str) -> np.ndarray:
    """Read a relation written in the tsv_to_bin layout, shape (rows, cols)."""
    with open(path + ".size") as f:
        rows = int(f.readline())
        cols = int(f.readline())
    data = np.fromfile(path, dtype="<u8", count=rows * cols)
    if data.size != rows * cols:
        raise IOError(f"{path}: expected {rows * cols} u64, found {data.size}")
    return data.reshape(rows, cols)


def write_empty_relation(path: str, arity: int = 2) -> None:
    write_relation(path, np.empty((0, arity + 1), dtype=np.uint64))
