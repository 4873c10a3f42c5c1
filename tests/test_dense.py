"""The dense row-closure evaluator (a transitive-closure-shaped SCC as one
breadth-first search per row in shared memory) gives what the hash-set path
and the oracle give: per-iteration history, final tuple sets, per-instance
results of batched waves."""
import numpy as np
import pytest

import oracle as O
import parallel_ra_b200 as P

pytestmark = pytest.mark.gpu


def run(rows, dense, program="tc"):
    """dense: the dense evaluator; otherwise the semi-naive hash-set path."""
    p = P.Program(0)
    if not dense:
        p.set_tuning(dense_max_bytes=0)
        p.set_evaluators(reach=False)
    rels = P.programs.PROGRAMS[program](p, rows)
    p.execute(1)
    return p, rels


def oracle_run(rows, program="tc"):
    o = O.OracleProgram()
    rels = P.programs.PROGRAMS[program](o, rows)
    o.execute(1)
    return o, rels


def er(n, m, seed):
    return P.datagen.with_row_ids(P.datagen.erdos_renyi(n, m, seed))


CASES = {
    "sparse": lambda: er(300, 450, 8),
    "dense_core": lambda: er(2000, 4000, 3),          # giant strongly connected core
    "config1": lambda: er(2000, 3000, 1),
    "cycle": lambda: np.array([[i, (i + 1) % 50, i] for i in range(50)], dtype=np.uint64),
    "self_loops_dups": lambda: np.array([[0, 0, 0], [0, 1, 1], [0, 1, 2], [1, 2, 3], [2, 0, 4], [3, 3, 5]],
                                        dtype=np.uint64),
    "long_path": lambda: np.stack([np.arange(699), np.arange(1, 700), np.arange(699)], axis=1).astype(np.uint64),
    "single_edge": lambda: np.array([[5, 9, 0]], dtype=np.uint64),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_dense_matches_hash_path_and_oracle(case):
    rows = CASES[case]()
    pd, rd = run(rows, True)
    assert pd.stats().dense_sccs == 1
    ph, rh = run(rows, False)
    assert ph.stats().dense_sccs == 0
    o, ro = oracle_run(rows)
    assert pd.history() == o.history() == ph.history()
    for name in ("T", "G"):
        a = pd.dump_full(rd[name])
        assert np.array_equal(a[:, :-1], o.dump_full(ro[name])[:, :-1]), name
        assert np.array_equal(a[:, :-1], ph.dump_full(rh[name])[:, :-1]), name
    ids = pd.dump_full(rd["T"])[:, -1]
    assert np.unique(ids).size == ids.size


def test_dense_is_deterministic_and_reruns():
    rows = er(1500, 2700, 5)
    p, r = run(rows, True)
    t1, h1 = p.dump_full(r["T"]), p.history()
    p.execute(1)
    assert p.history() == h1 and np.array_equal(p.dump_full(r["T"]), t1)
    q, rq = run(rows, True)
    assert np.array_equal(q.dump_full(rq["T"]), t1)


def test_dense_waves_match_plain_runs():
    insts = [er(int(n), int(m), 100 + i) for i, (n, m) in
             enumerate([(64, 60), (200, 390), (1000, 1900), (3000, 2500), (500, 1000), (40, 70)])]
    insts.append(np.empty((0, 3), dtype=np.uint64))
    w = P.batch.Runner("tc")
    got = w.run_wave(insts)
    assert w.prog.stats().dense_sccs == 1
    hashw = P.batch.Runner("tc")
    hashw.prog.set_tuning(dense_max_bytes=0)
    got_h = hashw.run_wave(insts)
    plain = P.batch.Runner("tc")
    for i, rows in enumerate(insts):
        want = plain.run_plain(rows)
        assert got[i].key() == want.key() == got_h[i].key(), i


def test_sg_and_reference_ids_keep_the_hash_path():
    p, _ = run(P.datagen.with_row_ids(P.datagen.random_tree(300, 2)), True, "sg")
    assert p.stats().dense_sccs == 0
    q = P.Program(0, id_order=P.engine.IDS_REFERENCE)
    P.programs.build_tc(q, er(300, 450, 8))
    q.execute(1)
    assert q.stats().dense_sccs == 0


def test_bitmap_join_with_deltas_beyond_the_candidate_buffer():
    """The TC join SCC on the device path with a bitmap seen set on T (the dense
    evaluator declined: the budget lies between the bitmap's and the evaluator's
    needs).  Its deltas reach tens of millions of tuples, far above the 4M-row
    candidate buffer, and feed the next iteration's join, whose look-back status
    array is sized by T's log.  History and tuples equal the dense evaluator's."""
    n = 16384
    rows = er(n, 2 * n, 12)
    pb = P.Program(0)
    pb.set_evaluators(reach=False)
    pb.set_tuning(dense_max_bytes=8 * n * (n // 32) + 4 * n)
    rb = P.programs.build_tc(pb, rows)
    pb.execute(1)
    st = pb.stats()
    assert st.dense_sccs == 0 and st.bitmap_relations >= 1
    pd, rd = run(rows, True)
    assert pd.stats().dense_sccs == 1
    hb = pb.history()
    assert hb == pd.history()
    assert max(d for _, pairs in hb for d, _ in pairs) > 1 << 22
    assert np.array_equal(pb.dump_full(rb["T"])[:, :-1], pd.dump_full(rd["T"])[:, :-1])
