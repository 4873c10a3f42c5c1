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


# ---------------------------------------------------------------------------
# programs read from a description (the generated analyses of the reference's
# tests/ directory, e.g. worstcase-110-terms-4-m.cpp; format in oracle/programs.h)
# ---------------------------------------------------------------------------

PREDICATES = {"true": 0, "false": 1, "eq": 2, "ne": 3, "lt": 4, "gt": 5, "le": 6, "ge": 7}
COPY_KINDS = {"copy": COPY, "acopy": ACOPY, "filter": COPY_FILTER}


def read_description(path: str) -> dict:
    """Parse a program description into relations, SCCs (add order), members,
    rules (per SCC, add order), dependencies and the batch size."""
    d = {"batch": 1, "relations": [], "sccs": [], "members": [], "rules": [], "deps": []}
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t or t[0].startswith("#"):
                continue
            k = t[0]
            if k == "batch":
                d["batch"] = int(t[1])
            elif k == "rel":
                d["relations"].append({"jcc": int(t[1]), "canonical": t[2] == "1", "arity": int(t[3]),
                                       "tag": int(t[4]), "version": FULL if t[5] == "FULL" else DELTA,
                                       "name": t[6], "file": None if t[7] == "-" else t[7]})
            elif k == "scc":
                d["sccs"].append({"fixpoint": t[1] == "1", "id": int(t[2])})
            elif k == "member":
                d["members"].append((int(t[1]), int(t[2]), t[3] == "1"))
            elif k == "join":
                d["rules"].append({"scc": int(t[1]), "kind": "join", "out": int(t[2]), "in0": int(t[3]),
                                   "ver0": FULL if t[4] == "FULL" else DELTA, "in1": int(t[5]),
                                   "ver1": FULL if t[6] == "FULL" else DELTA,
                                   "proj": [int(x) for x in t[7].split(",")]})
            elif k == "copy":
                d["rules"].append({"scc": int(t[1]), "kind": t[2], "out": int(t[3]), "in0": int(t[4]),
                                   "ver0": FULL if t[5] == "FULL" else DELTA, "pred": t[6],
                                   "proj": [int(x) for x in t[7].split(",")]})
            elif k == "dep":
                d["deps"].append((int(t[1]), int(t[2])))
    return d


def build_described(p, path: str, data_dir: str) -> dict:
    """Build a described program on ``p`` (engine or oracle), loading each
    relation's file from ``data_dir``; returns {relation name: handle} and
    stores the description's batch size under the key ``"__batch__"``."""
    from . import datagen
    d = read_description(path)
    handles = []
    out = {}
    for r in d["relations"]:
        h = p.relation(r["jcc"], r["arity"], r["tag"], r["name"], r["version"])
        rows = datagen.read_relation(f"{data_dir}/{r['file']}") if r["file"] else _empty(r["arity"])
        if rows.shape[1] != r["arity"] + 1:
            raise ValueError(f"{r['name']}: file has {rows.shape[1]} columns, relation {r['arity'] + 1}")
        p.load_rows(h, rows)
        handles.append(h)
        out[r["name"]] = h
    sccs = [p.scc(s["fixpoint"], s["id"]) for s in d["sccs"]]
    for s, r, init in d["members"]:
        p.add_relation(sccs[s], handles[r], init)
    for ru in d["rules"]:
        s = sccs[ru["scc"]]
        if ru["kind"] == "join":
            p.join(s, handles[ru["out"]], handles[ru["in0"]], ru["ver0"], handles[ru["in1"]], ru["ver1"], ru["proj"])
        else:
            p.copy(s, handles[ru["out"]], handles[ru["in0"]], ru["ver0"], ru["proj"], kind=COPY_KINDS[ru["kind"]],
                   pred=PREDICATES[ru["pred"]] if ru["kind"] == "filter" else 0)
    for a, b in d["deps"]:
        p.depend(sccs[a], sccs[b])
    out["__batch__"] = d["batch"]
    return out
