"""Batched execution: many independent instances of one program per launch.

A wave is one engine program over the disjoint union of its instances:
instance ``i``'s values are shifted by ``base[i]`` so that instances occupy
disjoint value ranges.  A join matches equal values only, so no derived tuple
mixes instances, and iteration ``k`` of the union performs iteration ``k`` of
every instance at once -- one CUDA graph launch (a WHILE-conditional graph per
fixed-point SCC) drives all of them.  The engine counts each iteration's new
tuples per instance inside its winner selection
(``ra_program_set_instances`` / ``ra_program_instance_history``) and
summarises every relation per instance with an order-independent digest of
the rebased data columns (``ra_relation_instance_summary``), so each instance
of a wave can be compared with a plain single-instance run of the same input:
same per-iteration delta sizes, same tuple count and digest per relation.

The reference has no batching: it runs one program instance per ``mpirun``
(tests/transitive_closure.cpp:46-87); a plain run here is that program on one
GPU (``Runner.run_plain``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .engine import Program, tuning_file
from .programs import PROGRAMS

# Device memory per derived tuple at the peak of a run (log keys + ids with
# growth slack, seen-set slots at the tuned load, candidate and loser-mark
# buffers) and the estimated derived tuples per wave: the autotuner's
# measurements when it has run on this machine, else conservative defaults.
_TUNED = tuning_file() or {}
BYTES_PER_TUPLE = float(_TUNED.get("bytes_per_tuple", 160.0))
WAVE_TUPLES = float(_TUNED.get("wave_tuples", 3e8))
# The engine's dense row-closure evaluator (transitive-closure-shaped SCCs):
# instances of at most DENSE_MAX_N values, bit matrices within DENSE_MAX_BYTES
# (ra_tuning.dense_max_bytes; a wave beyond it runs on the hash-set path).
DENSE_MAX_N = 65536
DENSE_MAX_BYTES = float((_TUNED.get("tuning") or {}).get("dense_max_bytes", 8e9))


def dense_bytes(span: int) -> float:
    """Device bytes of one instance's bit matrices (known + initial delta) and row counters."""
    return 2.0 * span * ((span + 31) // 32) * 4 + 16.0 * span


@dataclass
class InstanceResult:
    """What a run establishes about one instance."""
    counts: dict = field(default_factory=dict)    # relation -> rows of its full version
    digests: dict = field(default_factory=dict)   # relation -> data digest of those rows
    deltas: list = field(default_factory=list)    # per SCC: new tuples of each iteration before the fixpoint

    def key(self):
        return (tuple(sorted(self.counts.items())), tuple(sorted(self.digests.items())),
                tuple(tuple(d) for d in self.deltas))


def _mix64(k: np.ndarray) -> np.ndarray:
    """MurmurHash3's 64-bit finaliser (fmix64), elementwise on uint64."""
    k = k ^ (k >> np.uint64(33))
    k = k * np.uint64(0xFF51AFD7ED558CCD)
    k = k ^ (k >> np.uint64(33))
    k = k * np.uint64(0xC4CEB9FE1A85EC53)
    return k ^ (k >> np.uint64(33))


def data_digest(rows: np.ndarray, arity: int, base: int = 0) -> int:
    """Host restatement of the engine's per-instance digest of relation rows.

    Sum (mod 2^64) over rows of a hash of the data columns minus ``base``; the
    id column (if present) is ignored.  Equal to what
    ``ra_relation_instance_summary`` reports for the same rows.
    """
    if rows.shape[0] == 0:
        return 0
    with np.errstate(over="ignore"):
        h = np.full(rows.shape[0], (0x9E3779B97F4A7C15 * arity) & (2**64 - 1), dtype=np.uint64)
        for c in range(arity):
            col = rows[:, c].astype(np.uint64) - np.uint64(base)
            h = _mix64(h ^ (col + np.uint64((0x632BE59BD9B4E019 * (c + 1)) & (2**64 - 1))))
        return int(h.sum(dtype=np.uint64))


def _strip(seq):
    seq = [int(v) for v in seq]
    while seq and seq[-1] == 0:
        seq.pop()
    return seq


def value_span(rows: np.ndarray) -> int:
    """Values an instance occupies: 1 + its largest data value (at least 1)."""
    if rows.shape[0] == 0:
        return 1
    return int(rows[:, :-1].max()) + 1


def estimate_tuples(kind: str, rows: np.ndarray) -> float:
    """Expected derived tuples of an instance, for memory admission.

    ``tc`` on a random digraph with ``n`` nodes and mean out-degree ``d``:
    above ``d = 1`` a giant strongly connected core of ``s * n`` nodes reaches
    (and is reached by) about ``s * n`` nodes, ``s = 1 - exp(-d s)``, so the
    closure holds about ``(s n)^2`` pairs; below it a node reaches
    ``1 / (1 - d)`` nodes on average.  ``sg`` on a tree: pairs of nodes of the
    same depth, ``sum_l c_l^2`` over depth level sizes ``c_l``.
    """
    m = rows.shape[0]
    if m == 0:
        return 1.0
    if kind == "sg":
        parent = rows[:, 0].astype(np.int64)
        child = rows[:, 1].astype(np.int64)
        n = int(max(parent.max(), child.max())) + 1
        depth = np.zeros(n, dtype=np.int64)
        for _ in range(n):
            nd = depth.copy()
            nd[child] = depth[parent] + 1
            if np.array_equal(nd, depth):
                break
            depth = nd
        c = np.bincount(depth)
        return float((c.astype(np.float64) ** 2).sum()) + m
    n = value_span(rows)
    d = m / n
    if d > 1.0:
        s = 0.5
        for _ in range(100):
            s = 1.0 - math.exp(-d * s)
        return (s * n) ** 2 + 2.0 * n
    return n / max(1.0 - d, 1.0 / math.sqrt(n)) + m


def plan_waves(estimates, budget_tuples: float, max_values: int | None = None, spans=None,
               max_dense_bytes: float | None = None):
    """Split instance indices into waves whose estimated tuples stay within budget.

    Instances are taken in the given order; a wave closes when the next
    instance would overflow the budget (a single instance above it gets a wave
    of its own), or, with ``max_values``, the union's value range, or, with
    ``max_dense_bytes``, the bit matrices of the dense evaluator.
    """
    waves, cur, tot, vals, dense = [], [], 0.0, 0, 0.0
    for i, e in enumerate(estimates):
        sp = spans[i] if spans is not None else 0
        db = dense_bytes(sp) if max_dense_bytes is not None else 0.0
        if cur and (tot + e > budget_tuples or (max_values is not None and vals + sp > max_values)
                    or (max_dense_bytes is not None and dense + db > max_dense_bytes)):
            waves.append(cur)
            cur, tot, vals, dense = [], 0.0, 0, 0.0
        cur.append(i)
        tot += e
        vals += sp
        dense += db
    if cur:
        waves.append(cur)
    return waves


class Runner:
    """One engine program of a given kind, reused for every run it makes.

    ``run_plain`` runs one instance; ``run_wave`` runs many as one union
    program.  Reuse keeps device buffers and captured graphs across runs.
    """

    def __init__(self, kind: str, device: int = 0, id_order: int | None = None):
        if kind not in PROGRAMS:
            raise ValueError(f"unknown program {kind!r}")
        self.kind = kind
        self.prog = Program(device, id_order=id_order)
        self.rels = PROGRAMS[kind](self.prog, np.empty((0, 3), dtype=np.uint64))
        self.input = "G" if kind == "tc" else "edge"
        self._instances = None

    def close(self):
        self.prog.close()

    def _scc_blocks(self):
        """(scc_id, iterations) of the last run, in execution order."""
        return [(sid, len(pairs)) for sid, pairs in self.prog.history()]

    def run_plain(self, rows: np.ndarray) -> InstanceResult:
        if self._instances != 0:
            self.prog.set_instances([])
            self._instances = 0
        self.prog.load_rows(self.rels[self.input], rows)
        self.prog.execute()
        res = InstanceResult()
        for _, pairs in self.prog.history():
            res.deltas.append(_strip(p[0] for p in pairs))
        for name, h in self.rels.items():
            c, d = self.prog.instance_summary(h)
            res.counts[name] = int(c[0])
            res.digests[name] = int(d[0])
        return res

    @staticmethod
    def union_rows(rows_list):
        """(union rows, value bases): instance i's data columns shifted by base[i]."""
        k = len(rows_list)
        base = np.zeros(k, dtype=np.uint64)
        if not k:
            return np.empty((0, 3), dtype=np.uint64), base
        sizes = np.fromiter((r.shape[0] for r in rows_list), dtype=np.int64, count=k)
        union = np.concatenate(rows_list).astype(np.uint64, copy=False)
        # span of each instance: 1 + its largest data value (1 for an empty instance)
        spans = np.ones(k, dtype=np.uint64)
        nz = np.flatnonzero(sizes)
        if nz.size:
            row_max = union[:, 0].copy()
            for c in range(1, union.shape[1] - 1):
                np.maximum(row_max, union[:, c], out=row_max)
            starts = (np.cumsum(sizes) - sizes)[nz]
            spans[nz] = np.maximum.reduceat(row_max, starts) + np.uint64(1)
        if k > 1:
            base[1:] = np.cumsum(spans[:-1])
        shift = np.repeat(base, sizes)
        for c in range(union.shape[1] - 1):
            union[:, c] += shift
        return union, base

    def load_wave(self, rows_list) -> np.ndarray:
        """Rebase and concatenate the instances; declare them to the engine."""
        union, base = self.union_rows(rows_list)
        self.declare(base)
        self.prog.load_rows(self.rels[self.input], union)
        return base

    def declare(self, base):
        self.prog.set_instances(base)
        self._instances = len(base)

    def collect_wave(self, n: int) -> list[InstanceResult]:
        hist = self.prog.instance_history()
        out = [InstanceResult() for _ in range(n)]
        at = 0
        for _, iters in self._scc_blocks():
            blk = hist[at:at + iters]
            at += iters
            # per instance: rows up to its last non-zero count (its own iterations)
            nz = blk != 0
            last = np.where(nz.any(axis=0), iters - 1 - np.argmax(nz[::-1], axis=0), -1) if iters else \
                np.full(n, -1)
            cols = blk.T.tolist()
            for i in range(n):
                out[i].deltas.append(cols[i][:last[i] + 1])
        for name, h in self.rels.items():
            c, d = self.prog.instance_summary(h)
            c, d = c.tolist(), d.tolist()
            for i in range(n):
                out[i].counts[name] = c[i]
                out[i].digests[name] = d[i]
        return out

    def run_wave_resident(self, base, dev_rows: int, nrows: int) -> list[InstanceResult]:
        """A wave whose union rows (built by ``union_rows``) are already in device memory."""
        self.declare(base)
        self.prog.load_rows_device(self.rels[self.input], dev_rows, nrows)
        self.prog.execute()
        return self.collect_wave(len(base))

    def run_wave(self, rows_list) -> list[InstanceResult]:
        self.load_wave(rows_list)
        self.prog.execute()
        return self.collect_wave(len(rows_list))
