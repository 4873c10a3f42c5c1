"""Batched instances: a wave (one program over the rebased union of many
instances) gives every instance exactly what a plain single-instance run gives
-- per-iteration delta sizes, per-relation tuple counts and data digests -- and
what the oracle gives for that instance alone."""
import numpy as np
import pytest

import oracle as O
import parallel_ra_b200 as P
from parallel_ra_b200.batch import InstanceResult, data_digest, estimate_tuples, plan_waves, value_span


def small_instances(count, seed, n_lo=16, n_hi=600):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        m = int(round(rng.uniform(0.8, 2.0) * n))
        m = min(m, n * (n - 1))
        out.append(P.datagen.with_row_ids(P.datagen.erdos_renyi(n, m, seed * 7919 + i)))
    return out


def oracle_result(kind, rows):
    p = O.OracleProgram()
    rels = P.programs.PROGRAMS[kind](p, rows)
    p.execute(1)
    res = InstanceResult()
    for _, pairs in p.history():
        d = [a for a, _ in pairs]
        while d and d[-1] == 0:
            d.pop()
        res.deltas.append(d)
    for name, h in rels.items():
        full = p.dump_full(h)
        res.counts[name] = int(full.shape[0])
        res.digests[name] = data_digest(full, 2)
    p.close()
    return res


# ---------------------------------------------------------------- CPU-only


def test_data_digest_ignores_order_ids_and_base():
    rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(50, 80, 1))
    d0 = data_digest(rows, 2)
    perm = rows[np.random.default_rng(0).permutation(rows.shape[0])].copy()
    perm[:, 2] = 7
    assert data_digest(perm, 2) == d0
    shifted = rows.copy()
    shifted[:, :2] += np.uint64(1000)
    assert data_digest(shifted, 2, base=1000) == d0
    assert data_digest(rows[:-1], 2) != d0
    assert data_digest(rows[:0], 2) == 0


def test_plan_waves_budget_and_value_range():
    est = [5, 5, 20, 1, 1, 1, 30]
    waves = plan_waves(est, budget_tuples=10)
    assert waves == [[0, 1], [2], [3, 4, 5], [6]]
    assert sorted(i for w in waves for i in w) == list(range(len(est)))
    waves = plan_waves([1] * 6, budget_tuples=100, max_values=10, spans=[4] * 6)
    assert waves == [[0, 1], [2, 3], [4, 5]]


def test_estimates_track_oracle_sizes():
    """The admission estimate is within a small factor of the true closure size."""
    for inst in small_instances(6, 5, n_lo=200, n_hi=400):
        est = estimate_tuples("tc", inst)
        true = oracle_result("tc", inst).counts["T"]
        assert true / 8 <= est <= true * 8 + 4 * inst.shape[0], (est, true)


def test_union_principle_on_the_oracle():
    """The oracle run on the rebased union equals the per-instance runs: final
    sets split by value range, and the union's per-iteration delta sums."""
    insts = small_instances(4, 11)
    spans = [value_span(r) for r in insts]
    base = np.concatenate([[0], np.cumsum(spans[:-1])]).astype(np.uint64)
    union = np.concatenate([r + np.array([b, b, 0], dtype=np.uint64) for r, b in zip(insts, base)])
    p = O.OracleProgram()
    rels = P.programs.PROGRAMS["tc"](p, union)
    p.execute(1)
    full = p.dump_full(rels["T"])
    hist = p.history()
    singles = [oracle_result("tc", r) for r in insts]
    for i, (b, s) in enumerate(zip(base, singles)):
        hi = base[i + 1] if i + 1 < len(base) else np.uint64(2**63)
        mine = full[(full[:, 0] >= b) & (full[:, 0] < hi)]
        assert mine.shape[0] == s.counts["T"]
        assert data_digest(mine, 2, base=int(b)) == s.digests["T"]
    for blk, (_, pairs) in enumerate(hist):
        for k, (sd, _) in enumerate(pairs):
            assert sd == sum(s.deltas[blk][k] if k < len(s.deltas[blk]) else 0 for s in singles)
    p.close()


# ---------------------------------------------------------------- GPU


@pytest.mark.gpu
def test_tc_wave_matches_plain_and_oracle():
    insts = small_instances(48, 3)
    insts.append(np.empty((0, 3), dtype=np.uint64))                       # empty instance
    insts.append(np.array([[0, 1, 0]], dtype=np.uint64))                  # one edge
    insts.append(np.array([[0, 1, 0], [1, 0, 1], [1, 1, 2]], dtype=np.uint64))  # 2-cycle + self loop
    wave = P.batch.Runner("tc")
    got = wave.run_wave(insts)
    plain = P.batch.Runner("tc")
    for i, rows in enumerate(insts):
        want = plain.run_plain(rows)
        assert got[i].key() == want.key(), i
    for i in (0, 7, 48, 50):
        assert got[i].key() == oracle_result("tc", insts[i]).key(), i
    wave.close()
    plain.close()


def instance_rows(rows, base, i, arity):
    """Instance i's rows of a union relation dump: data columns in [base[i], base[i+1]),
    rebased to 0, in trie order (ids dropped: a wave numbers its ids across instances)."""
    lo = int(base[i])
    hi = int(base[i + 1]) if i + 1 < len(base) else 1 << 62
    d = rows[:, :arity].astype(np.int64)
    sel = (d[:, 0] >= lo) & (d[:, 0] < hi)
    out = d[sel] - lo
    return out[np.lexsort(out.T[::-1])] if out.shape[0] else out


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["tc", "sg"])
def test_wave_rows_equal_plain_runs(kind):
    """Row for row, every relation of every instance of a wave equals a plain single-instance run's."""
    if kind == "tc":
        insts = small_instances(24, 5)
    else:
        insts = [P.datagen.with_row_ids(P.datagen.random_tree(n, 300 + n)) for n in (3, 40, 200, 700)]
    wave = P.batch.Runner(kind)
    base = wave.load_wave(insts)
    wave.prog.execute()
    dumps = {name: wave.prog.dump_full(h) for name, h in wave.rels.items()}
    plain = P.batch.Runner(kind)
    for i, rows in enumerate(insts):
        plain.run_plain(rows)
        for name, h in plain.rels.items():
            want = plain.prog.dump_full(h)[:, :2].astype(np.int64)
            got = instance_rows(dumps[name], base, i, 2)
            assert np.array_equal(got, want), (i, name)
    wave.close()
    plain.close()


@pytest.mark.gpu
def test_sg_wave_matches_plain_and_oracle():
    insts = [P.datagen.with_row_ids(P.datagen.random_tree(n, 100 + n)) for n in (2, 17, 64, 200, 513, 1000)]
    got = P.batch.Runner("sg").run_wave(insts)
    plain = P.batch.Runner("sg")
    for i, rows in enumerate(insts):
        assert got[i].key() == plain.run_plain(rows).key(), i
        assert got[i].key() == oracle_result("sg", rows).key(), i


@pytest.mark.gpu
def test_sg_wave_with_large_deltas_matches_hash_path():
    """Same generation over trees of up to 16,384 nodes: about 10^8 tuples, with
    per-iteration deltas far above the 4M-row candidate buffer, through the
    instances' bitmap seen sets; the wave equals the hash-set wave and plain runs."""
    insts = [P.datagen.with_row_ids(P.datagen.random_tree(n, s)) for n, s in ((16384, 1), (8192, 3), (2000, 5))]
    w = P.batch.Runner("sg")
    got = w.run_wave(insts)
    assert w.prog.stats().bitmap_relations == 2          # TMP and SG of the recursive SCC
    h = P.batch.Runner("sg")
    h.prog.set_tuning(dense_max_bytes=0)
    got_h = h.run_wave(insts)
    assert h.prog.stats().bitmap_relations == 0
    plain = P.batch.Runner("sg")
    for i, rows in enumerate(insts):
        assert got[i].key() == got_h[i].key() == plain.run_plain(rows).key(), i
    assert max(max(d) for d in got[0].deltas if d) > 1 << 22
    for r in (w, h, plain):
        r.close()


@pytest.mark.gpu
def test_wave_in_reference_id_order():
    insts = small_instances(12, 9)
    got = P.batch.Runner("tc", id_order=P.engine.IDS_REFERENCE).run_wave(insts)
    plain = P.batch.Runner("tc")
    for i, rows in enumerate(insts):
        assert got[i].key() == plain.run_plain(rows).key(), i


@pytest.mark.gpu
def test_long_instance_grows_the_instance_matrix():
    """A 700-node path needs 699 iterations, past the initial 256 rows of the
    per-iteration instance counts: the iteration is replayed after the matrix grows."""
    n = 700
    path = np.stack([np.arange(n - 1), np.arange(1, n), np.arange(n - 1)], axis=1).astype(np.uint64)
    insts = [path] + small_instances(5, 21)
    got = P.batch.Runner("tc").run_wave(insts)
    assert got[0].counts["T"] == n * (n - 1) // 2
    assert len(got[0].deltas[1]) == n - 2
    plain = P.batch.Runner("tc")
    for i, rows in enumerate(insts):
        assert got[i].key() == plain.run_plain(rows).key(), i


@pytest.mark.gpu
def test_waves_reuse_one_program():
    insts = small_instances(30, 17)
    r = P.batch.Runner("tc")
    waves = plan_waves([estimate_tuples("tc", x) for x in insts], budget_tuples=2e5)
    assert len(waves) > 1
    got = {}
    for w in waves:
        for i, res in zip(w, r.run_wave([insts[i] for i in w])):
            got[i] = res
    plain = P.batch.Runner("tc")
    for i, rows in enumerate(insts):
        assert got[i].key() == plain.run_plain(rows).key(), i


@pytest.mark.gpu
def test_set_instances_rejects_unordered_bases():
    p = P.Program(0)
    with pytest.raises(P.RAError):
        p.set_instances([0, 5, 5])
    with pytest.raises(P.RAError):
        p.instance_history()
    p.close()


def test_plan_waves_respects_dense_bytes():
    from parallel_ra_b200.batch import dense_bytes
    spans = [1000, 1000, 1000, 5000]
    cap = 2.5 * dense_bytes(1000)
    waves = plan_waves([1, 1, 1, 1], budget_tuples=1e9, spans=spans, max_dense_bytes=cap)
    assert waves == [[0, 1], [2], [3]]


@pytest.mark.gpu
def test_tuple_across_instances_is_rejected():
    """An edge whose endpoints lie in different declared instances is a caller error:
    the run fails with RA_E_BADARG (no silent result, no out-of-range access)."""
    p = P.Program(0)
    rels = P.programs.build_tc(p, np.array([[0, 1, 0], [1, 2, 1], [3, 7, 2], [6, 5, 3]], dtype=np.uint64))
    p.set_instances([0, 5])
    with pytest.raises(P.RAError) as e:
        p.execute(1)
    assert e.value.status == P.engine.E_BADARG
