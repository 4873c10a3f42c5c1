"""The CPU oracle, pinned against golden vectors produced by the reference itself."""
import numpy as np
import pytest

import oracle as O
import parallel_ra_b200 as P
from conftest import GOLDEN_CASES, golden_input, load_golden, rows_digest

FAST = [c for c in GOLDEN_CASES if c not in ("er2000_tc",)]


@pytest.mark.parametrize("name", FAST)
def test_oracle_matches_reference_goldens(name):
    case = load_golden(name)
    rows = golden_input(case)
    assert rows_digest(rows) == case["input_sha256"]
    p = O.OracleProgram()
    rels = P.programs.PROGRAMS[case["program"]](p, rows)
    p.execute(1)
    assert [[sid, [list(x) for x in pairs]] for sid, pairs in p.history()] == case["history"]
    for rname, exp in case["relations"].items():
        got = p.dump_full(rels[rname])
        assert got.shape[0] == exp["count"]
        assert rows_digest(got) == exp["sha256"], rname
        if "rows" in exp:
            assert np.array_equal(got, np.array(exp["rows"], dtype=np.uint64).reshape(-1, exp["arity"] + 1))


def test_readme_fixture_counts():
    # README.md:21 (573 for g13236); g5955's chain of 4 edges closes to 10 pairs
    assert load_golden("g13236_tc")["relations"]["T"]["count"] == 573
    assert load_golden("g5955_tc")["relations"]["T"]["count"] == 10


def test_tc_delta_history_is_path_length_histogram():
    # Independent check: semi-naive TC adds, at iteration k, exactly the pairs whose
    # shortest path (shortest cycle for x == x) has length k + 1.
    e = P.datagen.erdos_renyi(300, 420, 9)
    n = 300
    adj = [[] for _ in range(n)]
    for u, v in e:
        adj[int(u)].append(int(v))
    hist = {}
    for s in range(n):
        dist = {s: 0}
        frontier = [s]
        d = 0
        selfd = None
        while frontier:
            d += 1
            nxt = []
            for u in frontier:
                for v in adj[u]:
                    if v == s and selfd is None:
                        selfd = d
                    if v not in dist:
                        dist[v] = d
                        nxt.append(v)
            frontier = nxt
        for v, dv in dist.items():
            if v != s:
                hist[dv] = hist.get(dv, 0) + 1
        if selfd is not None:
            hist[selfd] = hist.get(selfd, 0) + 1
    p = O.OracleProgram()
    P.programs.build_tc(p, P.datagen.with_row_ids(e))
    p.execute(1)
    (_, copy_hist), (_, join_hist) = p.history()
    assert copy_hist[0][0] == hist[1]
    deltas = [d for d, _ in join_hist]
    assert deltas == [hist.get(k, 0) for k in range(2, len(deltas) + 2)]
