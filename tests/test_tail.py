"""The tail kernel: small iterations back to back in one thread-block cluster.

Runs with the tail kernel (the default) and without it (RA_NO_TAIL=1) must give
the same log -- rows in the same order with the same intern ids -- and the same
history, and the tail kernel must actually have run iterations.  Transitive
closure (one join rule) on Erdos-Renyi graphs whose deltas shrink below and grow
above the cluster's size, same generation (two join rules) on the hash-set path,
and a long path whose every iteration is small.
"""
import os

import numpy as np
import pytest

import oracle as O
import parallel_ra_b200 as P


def as_lists(hist):
    return [[sid, [list(x) for x in pairs]] for sid, pairs in hist]


def run(program, rows, tail, **tuning):
    old = os.environ.get("RA_NO_TAIL")
    os.environ["RA_NO_TAIL"] = "0" if tail else "1"
    try:
        p = P.Program(0)
    finally:
        if old is None:
            del os.environ["RA_NO_TAIL"]
        else:
            os.environ["RA_NO_TAIL"] = old
    p.set_evaluators(reach=False, persistent=False)
    if tuning:
        p.set_tuning(**tuning)
    rels = P.programs.PROGRAMS[program](p, rows)
    p.execute(1)
    return p, rels


def compare(program, rows, out_rel, **tuning):
    a, ra = run(program, rows, True, **tuning)
    b, rb = run(program, rows, False, **tuning)
    sa, sb = a.stats(), b.stats()
    assert sa.tail_iterations > 0 and sb.tail_iterations == 0
    assert a.history() == b.history()
    for name in ra:
        assert np.array_equal(a.dump_full(ra[name]), b.dump_full(rb[name])), name
    got = a.dump_full(ra[out_rel])
    a.close()
    b.close()
    return got, sa


@pytest.mark.gpu
@pytest.mark.parametrize("n,m,seed", [(200_000, 190_000, 3), (1 << 20, 996_147, 5)])
def test_tc_with_and_without_the_tail_kernel(n, m, seed):
    rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(n, m, seed))
    _, st = compare("tc", rows, "T", dense_max_bytes=0.0)
    assert st.tail_iterations < st.iterations   # the large iterations stayed on the graph path


@pytest.mark.gpu
def test_tc_tail_kernel_against_the_oracle():
    rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(70_000, 69_000, 11))
    got, _ = compare("tc", rows, "T", dense_max_bytes=0.0)
    o = O.OracleProgram()
    orels = P.programs.build_tc(o, rows)
    o.execute(1)
    a, ra = run("tc", rows, True, dense_max_bytes=0.0)
    assert as_lists(a.history()) == as_lists(o.history())
    assert np.array_equal(got[:, :2], o.dump_full(orels["T"])[:, :2])
    a.close()


@pytest.mark.gpu
def test_sg_two_rules_on_the_hash_path():
    rows = P.datagen.with_row_ids(P.datagen.random_tree(3000, 9))
    compare("sg", rows, "SG", dense_max_bytes=0.0)


@pytest.mark.gpu
def test_long_path_every_iteration_in_the_tail():
    n = 3000
    e = np.stack([np.arange(n - 1), np.arange(1, n)], axis=1).astype(np.uint64)
    rows = P.datagen.with_row_ids(e)
    got, st = compare("tc", rows, "T", dense_max_bytes=0.0)
    assert got.shape[0] == n * (n - 1) // 2
    # all but the first iteration of each graph launch (one launch, plus one after each seen-set growth)
    assert st.tail_iterations >= st.iterations - 16
