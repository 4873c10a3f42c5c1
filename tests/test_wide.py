"""Wide tuples: programs whose tuples do not pack into one 63-bit key run with
every relation as rows of u64 columns in trie order.  The reference's own
generated analyses (tests/cfa-4-4-64.cpp, tests/worstcase-110-terms-4-m.cpp:
arity up to 23, joins on 0 to 16 columns, intern ids copied into data columns,
batch size 10) must give, relation by relation, the reference's rows including
intern ids, and its per-batch history; a synthetic program covers the rule
shapes one by one against the oracle."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import parallel_ra_b200 as P
from conftest import GOLDEN, ROOT, load_golden

GENERATED = ["cfa-4-4-64", "worstcase-110-terms-4-m"]


def digest(rows):
    return hashlib.sha256(np.ascontiguousarray(rows, dtype="<u8").tobytes()).hexdigest()


def run_described(p, prog):
    h = P.programs.build_described(p, os.path.join(GOLDEN, prog, "program.txt"), os.path.join(GOLDEN, prog, "data"))
    h["__batch__"] = batch = h.pop("__batch__")
    p.execute(batch)
    return h


def history_lists(p):
    return [[sid, [list(x) for x in pairs]] for sid, pairs in p.history()]


def check_against_golden(p, h, g):
    assert history_lists(p) == g["history"]
    for name, v in g["relations"].items():
        if name.startswith("__"):
            continue
        rows = p.dump_full(h[name])
        assert rows.shape[0] == v["count"], name
        assert digest(rows) == v["sha256"], name


# ---------------------------------------------------------------- CPU


def test_descriptions_parse():
    d = P.programs.read_description(os.path.join(GOLDEN, "worstcase-110-terms-4-m", "program.txt"))
    assert d["batch"] == 10
    assert (len(d["relations"]), len(d["sccs"]), len(d["rules"])) == (60, 19, 87)
    kinds = sorted({r["kind"] for r in d["rules"]})
    assert kinds == ["acopy", "copy", "filter", "join"]
    c = P.programs.read_description(os.path.join(GOLDEN, "cfa-4-4-64", "program.txt"))
    assert max(r["arity"] for r in c["relations"]) == 23
    assert min(r["jcc"] for r in c["relations"]) == 0


@pytest.mark.parametrize("prog", GENERATED)
def test_oracle_matches_reference_on_generated_programs(prog):
    o = O.OracleProgram()
    h = run_described(o, prog)
    check_against_golden(o, h, load_golden(prog))
    o.close()


# ---------------------------------------------------------------- GPU


@pytest.mark.gpu
@pytest.mark.parametrize("prog", GENERATED)
def test_wide_program_matches_reference(prog):
    p = P.Program(0)
    h = run_described(p, prog)
    check_against_golden(p, h, load_golden(prog))
    # a rerun of the same program starts from the loaded relations again
    hist = history_lists(p)
    p.execute(h["__batch__"])
    assert history_lists(p) == hist
    p.close()


@pytest.mark.gpu
def test_unchanged_generated_program_prints_the_reference_sizes(tmp_path):
    """tests/worstcase-110-terms-4-m.cpp of the reference, compiled unchanged against
    the C++ API layer, prints the sizes the reference prints after every SCC."""
    prog = "worstcase-110-terms-4-m"
    exe = os.path.join(ROOT, "parallel-ra_b200", "cxx", "bin", prog)
    assert os.path.exists(exe), "build the C++ programs (parallel-ra_b200/build.py) where the reference exists"
    (tmp_path / "data").mkdir()
    os.symlink(os.path.join(GOLDEN, prog, "data"), tmp_path / "data" / prog)
    (tmp_path / "run").mkdir()
    out = subprocess.run([exe], cwd=tmp_path / "run", capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if "total facts" in ln or ln.startswith("Total facts")]
    assert lines == load_golden(prog)["printed_sizes"]


BIG = 1 << 45   # two columns of 46 bits do not pack into 63


def build_shapes(p, seed):
    """Every rule shape of the wide path, on values above 2^45:
    copy (with a projected id), acopy (id into a data column), copy_filter,
    joins DELTA x FULL, FULL x DELTA, DELTA x DELTA, FULL x FULL and on zero columns."""
    rng = np.random.Generator(np.random.PCG64(seed))

    def rows(n, arity, lo, hi):
        data = rng.integers(lo, hi, size=(n, arity), dtype=np.uint64) + np.uint64(BIG)
        ids = np.arange(n, dtype=np.uint64) + np.uint64(7 << 40)
        return np.concatenate([data, ids[:, None]], axis=1)

    F = P.programs.FULL
    D = P.programs.DELTA
    E = p.relation(1, 2, 300, "E", F)
    T = p.relation(1, 2, 301, "T", F)
    I = p.relation(1, 2, 302, "I", F)
    P2 = p.relation(1, 3, 303, "P2", F)
    S = p.relation(0, 1, 304, "S", F)
    U = p.relation(0, 1, 305, "U", F)
    X = p.relation(2, 2, 306, "X", F)
    Fi = p.relation(1, 2, 307, "Fi", F)
    K = p.relation(1, 2, 308, "K", F)
    Q = p.relation(1, 2, 309, "Q", F)
    R = p.relation(1, 2, 301, "R", F)      # shares T's intern tag
    e = rows(150, 2, 0, 60)
    e = np.concatenate([e, e[:5]])          # duplicate rows in the file
    p.load_rows(E, e)
    p.load_rows(S, rows(3, 1, 0, 100))
    p.load_rows(U, rows(4, 1, 0, 100))
    p.load_rows(Q, rows(40, 2, 0, 25))
    for r in (T, I, P2, X, Fi, K, R):
        p.load_rows(r, np.empty((0, p._arity[r] + 1), dtype=np.uint64))

    s1 = p.scc(False, 1)
    p.add_relation(s1, E, False)
    p.add_relation(s1, T, True)
    p.copy(s1, T, E, F, [1, 0])
    s2 = p.scc(True, 2)                     # T(z, x) :- T(y, x), E(y, z); R mirrors it with the same tag
    p.add_relation(s2, E, False)
    p.add_relation(s2, T, True)
    p.add_relation(s2, R, False)
    p.join(s2, T, T, D, E, F, [3, 1])
    p.join(s2, R, E, F, T, D, [1, 3])       # FULL x DELTA: outer rows are T's delta
    s3 = p.scc(False, 3)
    p.add_relation(s3, T, False)
    p.add_relation(s3, I, True)
    p.copy(s3, I, T, F, [2, 0, 1], kind=P.programs.ACOPY)
    s4 = p.scc(False, 4)
    p.add_relation(s4, E, False)
    p.add_relation(s4, P2, True)
    p.join(s4, P2, E, F, E, F, [1, 0, 3])   # FULL x FULL
    s5 = p.scc(False, 5)
    p.add_relation(s5, S, False)
    p.add_relation(s5, U, False)
    p.add_relation(s5, X, True)
    p.join(s5, X, S, F, U, F, [0, 2])       # zero join columns: the cross product
    s6 = p.scc(False, 6)
    p.add_relation(s6, T, False)
    p.add_relation(s6, Fi, True)
    p.add_relation(s6, K, True)
    p.copy(s6, Fi, T, F, [0, 1], kind=P.programs.COPY_FILTER, pred=3)
    p.copy(s6, K, T, F, [0, 2])             # an intern id as a data column
    s7 = p.scc(True, 7)
    p.add_relation(s7, Q, True)
    p.join(s7, Q, Q, D, Q, D, [3, 0])       # DELTA x DELTA
    for a, b in ((s1, s2), (s2, s3), (s3, s6), (s4, s5)):
        p.depend(a, b)
    return {"E": E, "T": T, "I": I, "P2": P2, "S": S, "U": U, "X": X, "Fi": Fi, "K": K, "Q": Q, "R": R}


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [1, 3])
def test_wide_rule_shapes_match_the_oracle(batch):
    p = P.Program(0)
    rp = build_shapes(p, 5)
    p.execute(batch)
    o = O.OracleProgram()
    ro = build_shapes(o, 5)
    o.execute(batch)
    assert p.history() == o.history()
    for name in rp:
        a, b = p.dump_full(rp[name]), o.dump_full(ro[name])
        assert np.array_equal(a, b), name
    assert p.dump_full(rp["X"]).shape[0] == 12
    p.close()
    o.close()


def test_wide_rule_shapes_on_the_oracle_are_nontrivial():
    o = O.OracleProgram()
    ro = build_shapes(o, 5)
    o.execute(1)
    counts = {n: o.full_count(h) for n, h in ro.items()}
    assert counts["E"] == 150 and counts["X"] == 12 and counts["T"] > 150 and counts["I"] == counts["T"]
    assert counts["K"] == counts["T"] and counts["P2"] > 0 and counts["Q"] > 40 and counts["R"] > 0
    o.close()


@pytest.mark.gpu
def test_wide_equals_packed_at_scale():
    """TC on an ER graph of 20,000 nodes (452,970 closure tuples, dozens of iterations):
    with values lifted above 2^45 the program runs on the wide path; with the original
    values on the packed path in the reference's id order.  Histories, and every row
    with its intern id (values lowered back), agree."""
    rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(20000, 19000, 3))
    lifted = rows.copy()
    lifted[:, :2] += np.uint64(BIG)
    w = P.Program(0)
    rw = P.programs.build_tc(w, lifted)
    w.execute(1)
    k = P.Program(0, id_order=P.engine.IDS_REFERENCE)
    rk = P.programs.build_tc(k, rows)
    k.execute(1)
    assert w.history() == k.history()
    a, b = w.dump_full(rw["T"]), k.dump_full(rk["T"])
    a[:, :2] -= np.uint64(BIG)
    assert a.shape == b.shape and a.shape[0] > 400_000
    assert np.array_equal(a, b)
    w.close()
    k.close()


@pytest.mark.gpu
def test_wide_checkpoint_dumps(tmp_path):
    """Dumps after every batch of a wide program (the reference's layout: rows of
    arity + 1 u64 in trie order, per relation <name>_full / <name>_delta + .size) leave
    the results the reference's, and the last dump holds every relation's rows."""
    prog = "cfa-4-4-64"
    p = P.Program(0)
    p.set_checkpoint(str(tmp_path / "cp"), 1)
    h = run_described(p, prog)
    check_against_golden(p, h, load_golden(prog))
    dumps = os.listdir(tmp_path / "cp")
    hist = load_golden(prog)["history"]
    assert len(dumps) == sum(len(b[1]) for b in hist)
    # the last dump: the last batch of the last SCC (batch numbers restart with each SCC)
    last_scc = hist[-1][0]
    last = tmp_path / "cp" / max((d for d in dumps if d.startswith(f"checkpoint-{last_scc}-")),
                                 key=lambda d: int(d.split("-")[2]))
    for name, rel in h.items():
        if name.startswith("__"):
            continue
        parts = []
        for v in ("full", "delta"):
            f = last / f"{name}_{v}"
            if f.exists():
                parts.append(P.datagen.read_relation(str(f)))
        got = np.concatenate(parts) if parts else np.empty((0, p._arity[rel] + 1), dtype=np.uint64)
        want = p.dump_full(rel)
        assert np.array_equal(got[np.lexsort(got.T[::-1])], want), name
    p.close()


@pytest.mark.gpu
def test_wide_restart_from_own_dump(tmp_path):
    """TC on values above 2^45 (wide path): dump every 2 batches, restart from a dump in
    the middle of the fixpoint SCC; the copy SCC is not run again and the closure's
    tuples equal a straight run's."""
    rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(400, 600, 9))
    rows[:, :2] += np.uint64(BIG)
    p = P.Program(0)
    rels = P.programs.build_tc(p, rows)
    p.set_checkpoint(str(tmp_path / "cp"), 2)
    p.execute(1)
    want = p.dump_full(rels["T"])[:, :2]
    mids = sorted((int(d.split("-")[2]), d) for d in os.listdir(tmp_path / "cp") if d.startswith("checkpoint-1-"))
    dump = str(tmp_path / "cp" / mids[len(mids) // 2][1])
    assert open(os.path.join(dump, "scc_metadata")).read().split() == ["2"]
    q = P.Program(0)
    T = q.relation(1, 2, 257, "T", P.engine.FULL)
    G = q.relation(1, 2, 256, "G", P.engine.FULL)
    q.load_file(T, os.path.join(dump, "T_full"))
    q.load_file(G, os.path.join(dump, "G_full"))
    join = q.scc(True, 1)
    q.add_relation(join, G, False)
    q.add_relation(join, T, True)
    q.join(join, T, T, P.engine.DELTA, G, P.engine.FULL, [3, 1])
    copy = q.scc(False, 2)
    q.add_relation(copy, G, False)
    q.add_relation(copy, T, True)
    q.copy(copy, T, G, P.engine.FULL, [1, 0])
    q.depend(copy, join)
    q.set_restart(dump)
    q.execute(1)
    assert np.array_equal(q.dump_full(T)[:, :2], want)
    assert [sid for sid, _ in q.history()] == [1]
    p.close()
    q.close()
