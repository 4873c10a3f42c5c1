"""Transitive closure partitioned over P ranks, one process per GPU.

The reference scales by hash-partitioning every relation on its join columns
(src/relation/balanced_hash_relation.cpp:781), routing each new tuple to the
rank owning the hash of its head join columns (shmap_relation_exp.cpp:427-438)
with one MPI_Alltoallv per iteration (comm/all_to_allv_comm.cpp:113), and
testing the fixed point with an MPI_Allreduce of the delta sizes
(RAM/RA_tasks.cpp:1080-1081).

For the recursive rule of tests/transitive_closure.cpp,
    T(z, x) :- T_delta(y, x), G(y, z),
the head keeps column x of the recursive atom.  Partitioning T by a hash of
x -- rank r owns the rows whose source x hashes to r -- and replicating G makes
every derivation local: a rank's new tuples keep its own x, so nothing is
exchanged, and each rank runs its partition to its own fixed point on its own
GPU with the single-GPU engine.  Rank r's program is the TC program with the
copy SCC seeded from G_own (the edges whose source r owns) and G_own standing
for G in both SCCs' relation lists (G itself, replicated, is read by the join
as a fixed input).  Summed over ranks, every iteration's (sum |delta|, sum |full|)
pair is then the single-rank program's, and the closures' disjoint union is
its T; one reduction of the per-rank histories at the end (ranks that reached
their fixed point earlier contribute no new tuples and their final full
size) replaces the per-iteration all-reduce.  Exact for any P.

Programs whose recursive rules keep no column of the recursive atom (same
generation's two-way join) do not partition this way; they run as replicas.
"""
from __future__ import annotations

import numpy as np

from .programs import DELTA, FULL, _empty

_M1 = np.uint64(0xFF51AFD7ED558CCD)
_M2 = np.uint64(0xC4CEB9FE1A85EC53)


def owner(values: np.ndarray, world: int) -> np.ndarray:
    """Rank owning each value: a 64-bit finaliser hash of the value, modulo world."""
    k = np.asarray(values, dtype=np.uint64).copy()
    with np.errstate(over="ignore"):
        k ^= k >> np.uint64(33)
        k *= _M1
        k ^= k >> np.uint64(33)
        k *= _M2
        k ^= k >> np.uint64(33)
    return (k % np.uint64(world)).astype(np.int64)


def build_tc_partitioned(p, edge_rows: np.ndarray, rank: int, world: int) -> dict:
    """Rank ``rank``'s part of transitive closure over ``edge_rows`` (rows ``(src, dst, id)``)."""
    own = owner(edge_rows[:, 0], world) == rank
    T = p.relation(1, 2, 257, "T", FULL)
    G = p.relation(1, 2, 256, "G", FULL)
    GO = p.relation(1, 2, 258, "G_own", FULL)
    p.load_rows(T, _empty())
    p.load_rows(G, edge_rows)
    p.load_rows(GO, np.ascontiguousarray(edge_rows[own]))

    scc_join = p.scc(True, 1)
    p.add_relation(scc_join, GO, False)
    p.add_relation(scc_join, T, True)
    p.join(scc_join, T, T, DELTA, G, FULL, [3, 1])

    scc_copy = p.scc(False, 2)
    p.add_relation(scc_copy, GO, False)
    p.add_relation(scc_copy, T, True)
    p.copy(scc_copy, T, GO, FULL, [1, 0])

    p.depend(scc_copy, scc_join)
    return {"T": T, "G": G, "G_own": GO}


def combine_histories(histories: list) -> list:
    """The single-rank history from every rank's: per SCC (same order on every
    rank), per iteration, the sums of (sum |delta|, sum |full|); a rank past its
    fixed point adds (0, its last full size)."""
    out = []
    for blocks in zip(*histories):
        sid = blocks[0][0]
        assert all(b[0] == sid for b in blocks), "ranks ran their SCCs in different orders"
        L = max(len(b[1]) for b in blocks)
        pairs = [[0, 0] for _ in range(L)]
        for _, h in blocks:
            for k in range(L):
                d, f = h[k] if k < len(h) else (0, h[-1][1])
                pairs[k][0] += d
                pairs[k][1] += f
        out.append((sid, [tuple(x) for x in pairs]))
    return out


def global_history(local: list, group=None) -> list:
    """combine_histories across the ranks of a torch.distributed group (any backend):
    one all-gather of every rank's history, the same result on every rank."""
    import torch.distributed as dist
    gathered = [None] * dist.get_world_size(group)
    dist.all_gather_object(gathered, [(sid, [tuple(x) for x in h]) for sid, h in local], group=group)
    return combine_histories(gathered)
