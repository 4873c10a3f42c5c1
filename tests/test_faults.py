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
    p = P.Program(0)
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
