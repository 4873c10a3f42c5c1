"""Failure detection without a GPU fault: a device-side wait that runs out
reports RA_E_TIMEOUT and leaves the context usable; out-of-memory injected
through the allocator cap fails a run cleanly and the program (or the
server) recovers with exact results; corrupt relation metadata is rejected."""
import os

import numpy as np
import pytest

import oracle as O
import parallel_ra_b200 as P
from parallel_ra_b200.serve import Server, poisson_arrivals, request_mix, run_stream

pytestmark = pytest.mark.gpu


def tc_rows(n=600, m=900, seed=5):
    return P.datagen.with_row_ids(P.datagen.erdos_renyi(n, m, seed))


def test_bounded_wait_gives_up_and_context_stays_usable():
    assert P.engine.selftest_bounded_wait(0, 1 << 16) == P.engine.E_TIMEOUT
    assert P.engine.selftest_bounded_wait(0, 0) == P.engine.E_BADARG
    rows = tc_rows()
    p = P.Program(0)
    rels = P.programs.build_tc(p, rows)
    p.execute(1)
    o = O.OracleProgram()
    orels = P.programs.build_tc(o, rows)
    o.execute(1)
    assert p.history() == o.history()


@pytest.mark.parametrize("dense,where", [(True, "start"), (False, "start"), (False, "mid"), (True, "mid")])
def test_injected_out_of_memory_then_recovery(dense, where):
    """`start`: the cap stops the run while loading; `mid`: a cap of 60% of what the run
    holds at its peak stops it after the first SCC has run -- the next run must run every
    SCC again (the history holds both)."""
    rows = tc_rows(3000, 4500, 7)
    # the hash-set variant numbers ids in the reference's order: that path does not run an
    # iteration in slices, so a cap below its buffers fails the run (test_sliced_* covers slices)
    p = P.Program(0, id_order=None if dense else P.engine.IDS_REFERENCE)
    if not dense:
        p.set_tuning(dense_max_bytes=0)
    rels = P.programs.build_tc(p, rows)
    cap = 1 << 20                                    # far below what loading needs
    if where == "mid":
        p.execute(1)
        peak = p.stats().device_bytes_peak
        p.release()
        cap = int(0.6 * peak)
    p.set_memory_cap(cap)
    with pytest.raises(P.RAError) as e:
        p.execute(1)
    assert e.value.status == P.engine.E_OOM
    p.release()
    p.set_memory_cap(0)
    p.execute(1)                                     # the failed run left the program reusable
    o = O.OracleProgram()
    orels = P.programs.build_tc(o, rows)
    o.execute(1)
    assert p.history() == o.history()
    assert np.array_equal(p.dump_full(rels["T"])[:, :2], o.dump_full(orels["T"])[:, :2])


def test_server_recovers_from_out_of_memory_waves():
    """Every program capped far below its waves' needs: each wave fails, is retried alone
    (split while it does not fit) under the whole budget, and every result is exact."""
    reqs = request_mix(24, 17, large_share=0.0, n_hi=1500)
    server = Server(slots=2, budget_bytes=8e9, program_cap_bytes=2 << 20)
    run_stream(server, reqs, poisson_arrivals(len(reqs), 1e5, 3))
    server.close()
    assert server.oom_retries > 0
    plain = {"tc": P.batch.Runner("tc"), "sg": P.batch.Runner("sg")}
    for r in reqs:
        assert r.error is None
        assert r.result.key() == plain[r.kind].run_plain(r.rows).key(), r.rid


def test_corrupt_size_metadata_is_rejected(tmp_path):
    path = os.path.join(str(tmp_path), "edge")
    P.datagen.write_relation(path, tc_rows(50, 60, 1))
    p = P.Program(0)
    G = p.relation(1, 2, 256, "G", P.engine.FULL)
    with open(path + ".size", "w") as f:
        f.write("1000000000000\n3")                  # more rows than the file holds
    with pytest.raises(P.RAError) as e:
        p.load_file(G, path)
    assert e.value.status == P.engine.E_IO
    with open(path + ".size", "w") as f:
        f.write("60\n4")                             # wrong column count
    with pytest.raises(P.RAError):
        p.load_file(G, path)
    with open(path + ".size", "w") as f:
        f.write("garbage")
    with pytest.raises(P.RAError):
        p.load_file(G, path)
    os.remove(path + ".size")
    with pytest.raises(P.RAError):
        p.load_file(G, path)


def layered_graph(a, b, c):
    """Sources 0..a-1 -> every hub a..a+b-1 -> every target: one join iteration derives
    each (source, target) pair b times -- a * b * c candidates for a * c new tuples."""
    src = np.arange(a, dtype=np.uint64)
    hub = np.arange(a, a + b, dtype=np.uint64)
    tgt = np.arange(a + b, a + b + c, dtype=np.uint64)
    e1 = np.stack(np.meshgrid(src, hub, indexing="ij"), axis=-1).reshape(-1, 2)
    e2 = np.stack(np.meshgrid(hub, tgt, indexing="ij"), axis=-1).reshape(-1, 2)
    return P.datagen.with_row_ids(np.concatenate([e1, e2]))


def test_sliced_iteration_under_a_memory_cap():
    """An iteration whose candidates (9M: 216 MB of candidate buffer and marks at the
    engine's 2x growth) exceed what the cap leaves -- 100 MB below the uncapped run's
    peak -- runs in slices of outer rows: same history and tuples as the oracle, and
    the same log, ids included, as the uncapped run."""
    rows = layered_graph(300, 100, 300)
    o = O.OracleProgram()
    orels = P.programs.build_tc(o, rows)
    o.execute(1)

    def run(cap):
        p = P.Program(0)
        p.set_tuning(dense_max_bytes=0)   # the hash-set path (the dense evaluator would take 700 values)
        p.set_evaluators(reach=False)
        p.set_memory_cap(cap)
        rels = P.programs.build_tc(p, rows)
        p.execute(1)
        return p, rels

    free, fr = run(0)
    cap = free.stats().device_bytes_peak - (100 << 20)
    capped, cr = run(cap)
    st = capped.stats()
    assert st.sliced_iterations >= 1 and st.sliced_passes >= 2
    assert st.device_bytes_peak <= cap
    assert capped.history() == o.history()
    got = capped.dump_full(cr["T"])
    assert np.array_equal(got[:, :2], o.dump_full(orels["T"])[:, :2])
    assert np.array_equal(got, free.dump_full(fr["T"]))   # the same log, ids included
    assert free.stats().sliced_iterations == 0

