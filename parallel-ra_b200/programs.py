"""Datalog programs expressed through the builder methods of a program object.

A builder is any object with ``relation / load_rows / scc / add_relation /
join / copy / depend`` (the B200 engine binding ``engine.Program`` has them).
The rule sets are those of the C++ programs:

* ``tc``: tests/transitive_closure.cpp:56-77 of parallel-RA -- ``T`` stored as
  ``(dst, src)``; SCC 2 copies ``G`` FULL with ``{1, 0}``; SCC 1 joins
  ``T`` DELTA with ``G`` FULL and projects ``{3, 1}`` until no new tuple.
* ``sg``: same generation over parent->child edges (base join + filtering
  copy ``x != y``, then a two-join recursive SCC through ``TMP``).
"""
from __future__ import annotations

import numpy as np

DELTA, FULL = 0, 1
COPY, ACOPY, COPY_FILTER = 0, 1, 2
PRED_NE = 3


def _empty(arity=2):
    return np.empty((0, arity + 1), dtype=np.uint64)


def build_tc(p, edge_rows: np.ndarray) -> dict:
    """Transitive closure over ``edge_rows`` (rows ``(src, dst, id)``)."""
    T = p.relation(1, 2, 257, "T", FULL)
    G = p.relation(1, 2, 256, "G", FULL)
    p.load_rows(T, _empty())
    p.load_rows(G, edge_rows)

    scc_join = p.scc(True, 1)
    p.add_relation(scc_join, G, False)
    p.add_relation(scc_join, T, True)
    p.join(scc_join, T, T, DELTA, G, FULL, [3, 1])

    scc_copy = p.scc(False, 2)
    p.add_relation(scc_copy, G, False)
    p.add_relation(scc_copy, T, True)
    p.copy(scc_copy, T, G, FULL, [1, 0])

    p.depend(scc_copy, scc_join)
    return {"T": T, "G": G}


def build_sg(p, edge_rows: np.ndarray) -> dict:
    """Same generation over ``edge_rows`` (rows ``(parent, child, id)``)."""
    E = p.relation(1, 2, 300, "edge", FULL)
    SGB = p.relation(1, 2, 301, "SGB", FULL)
    SG = p.relation(1, 2, 302, "SG", FULL)
    TMP = p.relation(1, 2, 303, "TMP", FULL)
    p.load_rows(E, edge_rows)
    for r in (SGB, SG, TMP):
        p.load_rows(r, _empty())

    base = p.scc(False, 10)
    p.add_relation(base, E, False)
    p.add_relation(base, SGB, True)
    p.join(base, SGB, E, FULL, E, FULL, [1, 3])

    filt = p.scc(False, 11)
    p.add_relation(filt, SGB, False)
    p.add_relation(filt, SG, True)
    p.copy(filt, SG, SGB, FULL, [0, 1], kind=COPY_FILTER, pred=PRED_NE)

    rec = p.scc(True, 12)
    p.add_relation(rec, E, False)
    p.add_relation(rec, SG, True)
    p.add_relation(rec, TMP, False)
    p.join(rec, TMP, SG, DELTA, E, FULL, [1, 3])
    p.join(rec, SG, TMP, DELTA, E, FULL, [1, 3])

    p.depend(base, filt)
    p.depend(filt, rec)
    return {"edge": E, "SGB": SGB, "SG": SG, "TMP": TMP}


PROGRAMS = {"tc": build_tc, "sg": build_sg}
