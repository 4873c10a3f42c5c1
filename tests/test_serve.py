"""Serving: admission logic (CPU) and continuous batching whose every result
equals the request's plain single-instance run (GPU)."""
import numpy as np
import pytest

import parallel_ra_b200 as P
from parallel_ra_b200.serve import Request, Server, poisson_arrivals, request_mix, run_stream


def fake(rid, kind, est, span=100):
    return Request(rid, kind, np.empty((0, 3), dtype=np.uint64), est_tuples=est, span=span)


def test_admission_takes_oldest_kind_in_order_within_budget():
    s = Server(slots=2, budget_bytes=1000, wave_tuples=50, bytes_per_tuple=10, start=False)
    for r in (fake(0, "tc", 20), fake(1, "sg", 5), fake(2, "tc", 20), fake(3, "tc", 20), fake(4, "sg", 5)):
        s._queue.append(r)
    kind, picked, est = s._take_wave(0)
    assert kind == "tc" and [r.rid for r in picked] == [0, 2]          # 60 tuples would pass wave_tuples=50
    assert s._used[0] == 400 and s._busy[0]
    kind, picked, _ = s._take_wave(1)
    assert kind == "sg" and [r.rid for r in picked] == [1, 4]
    assert [r.rid for r in s._queue] == [3]
    # worker 0 finishes holding 300 bytes; worker 1 still runs with 100 charged
    s._busy[0], s._used[0] = False, 300
    s._queue.appendleft(fake(5, "tc", 95))                              # 950 bytes > 1000 - 100
    assert s._take_wave(0) is None                                      # waits for the running wave
    s._busy[1], s._used[1] = False, 100                                 # nothing runs: idle buffers are released
    kind, picked, _ = s._take_wave(0)
    assert [r.rid for r in picked] == [5] and s._used[1] == 0


def test_oversized_request_runs_alone_when_nothing_else_runs():
    s = Server(slots=1, budget_bytes=100, wave_tuples=1e9, bytes_per_tuple=10, start=False)
    s._queue.extend([fake(0, "tc", 50), fake(1, "tc", 1)])
    kind, picked, _ = s._take_wave(0)
    assert [r.rid for r in picked] == [0]


def test_request_mix_and_arrivals():
    reqs = request_mix(400, 3, large_n=1 << 10)
    kinds = [r.kind for r in reqs]
    assert 0.1 < kinds.count("sg") / len(reqs) < 0.3
    a = poisson_arrivals(20000, 1000.0, 1)
    assert np.all(np.diff(a) > 0) and abs(a[-1] - 20.0) < 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("rate,slots", [(1e5, 3), (300.0, 2)])
def test_served_results_equal_plain_runs(rate, slots):
    reqs = request_mix(160, 11, large_n=1 << 12, n_hi=1500)
    server = Server(slots=slots, budget_bytes=20e9)
    stats = run_stream(server, reqs, poisson_arrivals(len(reqs), rate, 5))
    server.close()
    assert stats["requests"] == len(reqs)
    plain = {"tc": P.batch.Runner("tc"), "sg": P.batch.Runner("sg")}
    for r in reqs:
        assert r.result.key() == plain[r.kind].run_plain(r.rows).key(), r.rid
    if rate > 1e4:
        assert max(w.size for w in server.waves) > 1                     # requests were batched
        spans = sorted((w.start, w.end, w.worker) for w in server.waves)
        assert any(b[0] < a[1] and b[2] != a[2] for a, b in zip(spans, spans[1:]))   # waves overlapped


@pytest.mark.gpu
def test_small_budget_forces_many_waves_and_stays_exact():
    reqs = request_mix(40, 13, large_share=0.0, n_hi=1500)
    server = Server(slots=2, budget_bytes=2e8, bytes_per_tuple=200)
    run_stream(server, reqs, poisson_arrivals(len(reqs), 1e5, 2))
    server.close()
    assert len(server.waves) > 5
    plain = {"tc": P.batch.Runner("tc"), "sg": P.batch.Runner("sg")}
    for r in reqs:
        assert r.result.key() == plain[r.kind].run_plain(r.rows).key(), r.rid


def test_oom_retry_waits_for_others_and_runs_alone():
    """Two workers that both ran out of memory retry one after the other, each alone."""
    import threading
    s = Server(slots=2, budget_bytes=1000, start=False)
    order = []

    class FakeRunner:
        def __init__(self, w):
            self.w = w
            self.prog = type("P", (), {"release": lambda self_: None})()

        def run_wave(self, rows):
            order.append(("start", self.w, tuple(s._busy)))
            order.append(("end", self.w))
            return ["ok"] * len(rows)
    s._runners = [{"tc": FakeRunner(0)}, {"tc": FakeRunner(1)}]
    s._busy = [True, True]
    out = {}

    def worker(w):             # what Server._work does around a retry: the wave ends, the worker is idle
        out[w] = s._retry_alone(w, s._runners[w]["tc"], [fake(w, "tc", 1)])
        with s._cv:
            s._busy[w] = False
            s._cv.notify_all()
    ts = [threading.Thread(target=worker, args=(w,), daemon=True) for w in (0, 1)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(10)
    assert out == {0: ["ok"], 1: ["ok"]}
    starts = [e for e in order if e[0] == "start"]
    assert len(starts) == 2
    for _, w, busy in starts:                  # nobody else was busy while a retry ran
        assert not busy[1 - w]
    assert s._exclusive is None and s.oom_retries == 2


def test_large_tc_requests_wave_apart_from_dense_ones():
    s = Server(slots=1, budget_bytes=1e12, wave_tuples=1e9, bytes_per_tuple=1, start=False)
    s._queue.extend([fake(0, "tc", 1), fake(1, "tc", 1, span=1 << 18), fake(2, "tc", 1), fake(3, "tc", 1, span=1 << 18)])
    _, picked, _ = s._take_wave(0)
    assert [r.rid for r in picked] == [0, 2]
    s._busy[0] = False
    _, picked, _ = s._take_wave(0)
    assert [r.rid for r in picked] == [1, 3]


def test_worker_failure_names_the_wave_and_stops_the_workers():
    """A wave that fails with an engine error (not out of memory) ends the stream:
    drain() raises, the failed wave's worker, kind and request ids are recorded, and
    every worker thread has stopped before the error reaches the caller."""
    s = Server(slots=2, budget_bytes=1e9, start=False)

    class FailingRunner:
        prog = None

        def run_wave(self, rows):
            raise P.RAError(1, "bad argument")

        def close(self):
            pass
    s._runners = [{"tc": FailingRunner()}, {"tc": FailingRunner()}]
    for t in s._workers:
        t.start()
    s.submit(fake(7, "tc", 10))
    with pytest.raises(RuntimeError):
        s.drain(1, timeout=10)
    assert len(s.failed_waves) == 1
    w, kind, rids = s.failed_waves[0]
    assert kind == "tc" and rids == [7] and w in (0, 1)
    assert not any(t.is_alive() for t in s._workers)
