"""ra_rows_distinct_noalloc: the relation-loading sort + distinct for callers
that cannot allocate device memory (fixed static scratch instead of cudaMalloc).

Checked against the allocating path that computes the same rows: load the
rows into a relation, run the program, dump the relation's full version.
This file is collected last on purpose; it passes alone and after the suite.
"""
import ctypes

import numpy as np
import pytest

import parallel_ra_b200 as P

MAX_ROWS = 1 << 17


def test_rejects_more_rows_than_the_scratch_holds():
    L = P.engine.lib()
    st = L.ra_rows_distinct_noalloc(None, MAX_ROWS + 1, 2, None, None, None)
    assert st == 1   # RA_E_BADARG, before touching any device


def rows_with_duplicates(n, arity, seed, vmax):
    rng = np.random.default_rng(seed)
    base = rng.integers(0, vmax, size=(max(n // 2, 1), arity + 1), dtype=np.uint64)
    base[:, -1] = rng.integers(0, 2**63, size=base.shape[0], dtype=np.uint64)
    pick = rng.integers(0, base.shape[0], size=n)
    rows = base[pick].copy()
    # some rows share data columns but carry their own id
    alt = rng.random(n) < 0.1
    rows[alt, -1] = rng.integers(0, 2**63, size=int(alt.sum()), dtype=np.uint64)
    return rows


def distinct_via_program(rows, arity):
    p = P.Program(0)
    r = p.relation(1, arity, 1, "R")
    p.load_rows(r, rows)
    p.execute(1)
    return p.dump_full(r)


def distinct_noalloc(rows, arity):
    import torch
    dev_in = torch.from_numpy(rows.view(np.int64)).cuda()
    dev_out = torch.full_like(dev_in, -1)
    dev_n = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    L = P.engine.lib()
    st = L.ra_rows_distinct_noalloc(dev_in.data_ptr(), rows.shape[0], arity, dev_out.data_ptr(), dev_n.data_ptr(),
                                    None)
    assert st == 0, P.engine.lib().ra_status_string(st)
    torch.cuda.synchronize()
    m = int(dev_n.item())
    return dev_out.cpu().numpy().view(np.uint64)[:m]


@pytest.mark.gpu
def test_noalloc_matches_relation_loading_twice_in_a_row():
    cases = [(MAX_ROWS, 2, 11, 1 << 20), (5000, 3, 12, 300)]
    for n, arity, seed, vmax in cases:
        rows = rows_with_duplicates(n, arity, seed, vmax)
        want = distinct_via_program(rows, arity)
        got = distinct_noalloc(rows, arity)
        assert got.shape == want.shape
        assert np.array_equal(got, want)


@pytest.mark.gpu
def test_noalloc_zero_rows_and_unpackable_rows():
    import torch
    L = P.engine.lib()
    out = torch.full((4, 3), -7, dtype=torch.int64, device="cuda")
    n = torch.full((1,), 99, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    assert L.ra_rows_distinct_noalloc(None, 0, 2, out.data_ptr(), n.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert int(n.item()) == 0
    assert bool((out == -7).all())   # nothing written
    # three columns of values near 2^40 need 3 x 41 bits: more than one packed key holds
    rows = np.array([[1 << 40, 1, 2, 0], [3, 1 << 40, 5, 1]], dtype=np.uint64)
    dev_in = torch.from_numpy(rows.view(np.int64)).cuda()
    torch.cuda.synchronize()
    st = L.ra_rows_distinct_noalloc(dev_in.data_ptr(), 2, 3, out.data_ptr(), n.data_ptr(), None)
    torch.cuda.synchronize()
    assert st == 5   # RA_E_UNSUPPORTED
    assert bool((out == -7).all())

