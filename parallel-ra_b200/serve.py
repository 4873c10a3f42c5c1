"""Serving: continuous batching of independent program instances on one GPU.

Requests (a program kind -- ``tc`` or ``sg`` -- and its input rows) arrive
over time.  ``slots`` worker threads each own one engine program per kind (its
own CUDA stream and device buffers).  A free worker forms a wave from what has
arrived by then: the oldest waiting request fixes the kind, and further
waiting requests of that kind join in arrival order while the wave's memory
estimate fits the admission budget.  The wave runs as one program over the
rebased union of its instances (``batch.Runner``); the workers' waves overlap
on the device, and requests that arrive meanwhile wait for the next free
worker -- continuous batching, not a queue served one instance at a time.

Admission.  A request's device-memory estimate is its expected derived tuples
(``batch.estimate_tuples``, a growth model of the closure from the input's
size and degree, or depth profile for ``sg``) times the device bytes per
derived tuple the autotuner measured, times a per-kind correction learnt from
completed waves (realised tuples / estimated tuples, from the per-instance
delta counts the engine reports).  The sum over running waves of
max(estimate, memory the worker's program already holds) stays within
``budget_bytes``; a worker whose idle program holds more than its share of the
budget releases it (``ra_program_release``).

Every request's result (per-iteration delta sizes, per-relation counts and
data digests) is what a plain single-instance run gives: the wave construction
never mixes instances (see ``batch``), which tests/test_serve.py checks.
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass

import numpy as np

from . import batch
from .batch import DENSE_MAX_BYTES, DENSE_MAX_N, Runner, dense_bytes, estimate_tuples, value_span
from .engine import E_OOM, RAError


@dataclass
class Request:
    rid: int
    kind: str
    rows: np.ndarray
    arrival: float = 0.0              # seconds after the stream's start (scheduled)
    est_tuples: float = 0.0
    span: int = 0                     # values the instance occupies
    submitted: float | None = None    # perf_counter at submission
    started: float | None = None      # its wave's start
    done: float | None = None         # its wave's end (results available)
    wave: int | None = None
    result: batch.InstanceResult | None = None
    error: str | None = None

    @property
    def latency(self) -> float | None:
        return None if self.done is None or self.submitted is None else self.done - self.submitted


@dataclass
class WaveRecord:
    wave: int
    kind: str
    worker: int
    size: int
    est_tuples: float
    tuples: int
    start: float
    end: float
    held_bytes: int
    launches: int = 0


class Server:
    def __init__(self, device: int = 0, slots: int = 4, budget_bytes: float = 150e9,
                 wave_tuples: float | None = None, bytes_per_tuple: float | None = None,
                 max_wave_requests: int = 8192, program_cap_bytes: float | None = None, start: bool = True):
        self.device = device
        self.slots = slots
        self.budget = float(budget_bytes)
        b = float(bytes_per_tuple or batch.BYTES_PER_TUPLE)
        # a wave at most the tuned size, and at most one slot's share of the budget
        self.wave_tuples = float(wave_tuples or min(batch.WAVE_TUPLES, self.budget / (slots * b)))
        self.bpt = {"tc": b, "sg": b}               # device bytes per derived output tuple, learnt per kind
        self.max_wave_requests = max_wave_requests
        # optional hard cap per program (ra_program_set_memory_cap): a wave past it fails fast with
        # out of memory instead of growing into other workers' share; its retry alone is capped
        # by the whole budget only
        self.program_cap = int(program_cap_bytes) if program_cap_bytes else 0
        self.correction = {"tc": 1.0, "sg": 1.0}    # realised / estimated output tuples, learnt per kind
        self._queue: collections.deque[Request] = collections.deque()
        self._cv = threading.Condition()
        self._used = [0.0] * slots           # bytes charged by each worker (running wave or held buffers)
        self._busy = [False] * slots
        self._exclusive = None               # worker retrying a wave alone after running out of memory
        self.oom_retries = 0
        self._stop = False
        self._wave_id = 0
        self.waves: list[WaveRecord] = []
        self.completed: list[Request] = []
        self._workers = [threading.Thread(target=self._work, args=(i,), daemon=True) for i in range(slots)]
        self._runners: list[dict] = [dict() for _ in range(slots)]
        self._errors: list[BaseException] = []
        self.failed_waves: list[tuple] = []  # (worker, kind, request ids) of waves that raised
        if start:
            for t in self._workers:
                t.start()

    # ------------------------------------------------------------------ client side
    def submit(self, req: Request) -> None:
        if not req.est_tuples:
            req.est_tuples = estimate_tuples(req.kind, req.rows)
        if not req.span:
            req.span = value_span(req.rows)
        req.submitted = time.perf_counter()
        with self._cv:
            self._queue.append(req)
            self._cv.notify()

    def drain(self, expected: int, timeout: float = 600.0) -> None:
        """Wait until ``expected`` requests have completed (or a worker failed)."""
        deadline = time.perf_counter() + timeout
        with self._cv:
            while len(self.completed) < expected and not self._errors:
                left = deadline - time.perf_counter()
                if left <= 0:
                    raise TimeoutError(f"{len(self.completed)} of {expected} requests completed")
                self._cv.wait(min(left, 0.5))
        if self._errors:
            self.close()   # stop and join the workers before the failure propagates
            raise RuntimeError("a serving worker failed") from self._errors[0]

    def close(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._workers:
            if t.is_alive():
                t.join()
        for rs in self._runners:
            for r in rs.values():
                r.close()

    # ------------------------------------------------------------------ workers
    @staticmethod
    def _cls(req: Request):
        """Requests that share a wave: same program, and for ``tc`` the same side of
        the dense evaluator's size limit (one large instance would send the
        whole wave to the hash-set path)."""
        return req.kind, req.kind == "tc" and req.span <= DENSE_MAX_N

    def _mem(self, req: Request) -> float:
        return req.est_tuples * self.correction[req.kind] * self.bpt[req.kind]

    def _release_idle(self, w: int) -> None:
        """Free the buffers idle workers' programs hold (lock held: an idle worker
        touches its programs only after taking a wave under the lock)."""
        for i in range(self.slots):
            if i != w and not self._busy[i] and self._used[i] > 0:
                for r in self._runners[i].values():
                    r.prog.release()
                self._used[i] = 0.0

    def _take_wave(self, w: int):
        """Pop the next wave for worker w (called with the lock held); None if nothing fits now."""
        if not self._queue or (self._exclusive is not None and self._exclusive != w):
            return None
        kind = self._queue[0].kind
        cls = self._cls(self._queue[0])
        dense_cap = 0.9 * DENSE_MAX_BYTES if cls[1] else None
        held = self._used[w]
        first = self._mem(self._queue[0])
        others = sum(u for i, u in enumerate(self._used) if i != w)
        if max(held, first) > self.budget - others:
            if any(self._busy[i] for i in range(self.slots) if i != w):
                return None            # the oldest request waits for memory of running waves
            self._release_idle(w)      # only idle buffers stand in the way
            others = 0.0
        free = self.budget - others
        picked, est, mem, dense = [], 0.0, 0.0, 0.0
        for req in self._queue:
            if self._cls(req) != cls:
                continue
            m = self._mem(req)
            e = req.est_tuples * self.correction[kind]
            db = dense_bytes(req.span) if dense_cap is not None else 0.0
            if picked and (est + e > self.wave_tuples or max(held, mem + m) > free
                           or len(picked) >= self.max_wave_requests
                           or (dense_cap is not None and dense + db > dense_cap)):
                break
            picked.append(req)         # the first one always (alone it may exceed an empty budget)
            est += e
            mem += m
            dense += db
        taken = set(id(r) for r in picked)
        self._queue = collections.deque(r for r in self._queue if id(r) not in taken)
        self._used[w] = max(held, mem)
        self._busy[w] = True
        return kind, picked, est

    def _runner(self, w: int, kind: str) -> Runner:
        rs = self._runners[w]
        if kind not in rs:
            rs[kind] = Runner(kind, self.device)
            if self.program_cap:
                rs[kind].prog.set_memory_cap(self.program_cap)
        return rs[kind]

    def _work(self, w: int) -> None:
        current = None
        try:
            while True:
                with self._cv:
                    job = None
                    while job is None:
                        if self._stop:
                            return
                        job = self._take_wave(w)
                        if job is None:
                            self._cv.wait(0.05)
                    kind, reqs, est = job
                    current = (w, kind, [r.rid for r in reqs])
                    wid = self._wave_id
                    self._wave_id += 1
                runner = self._runner(w, kind)
                t0 = time.perf_counter()
                for r in reqs:
                    r.started = t0
                try:
                    out = runner.run_wave([r.rows for r in reqs])
                except RAError as e:
                    if e.status != E_OOM:
                        raise
                    out = self._retry_alone(w, runner, reqs)
                t1 = time.perf_counter()
                tuples = sum(sum(o.counts.values()) for o in out if o is not None)
                st = runner.prog.stats()
                held = st.device_bytes
                # realised growth (the instances' delta counts add up to their output sizes)
                # corrects the next admissions of this kind: tuples per estimate, bytes per tuple
                real = sum(o.counts[self._output(kind)] for o in out if o is not None)
                raw = sum(r.est_tuples for r in reqs)
                with self._cv:
                    ratio = min(max(real / max(raw, 1.0), 0.5), 8.0)
                    self.correction[kind] = max(0.7 * self.correction[kind] + 0.3 * ratio, 0.75)
                    if real > 1_000_000:
                        self.bpt[kind] = max(0.7 * self.bpt[kind] + 0.3 * st.device_bytes_peak / real, 32.0)
                    for r, o in zip(reqs, out):
                        r.result = o
                        r.done = t1
                        r.wave = wid
                        if o is None:
                            r.error = "out of device memory even alone on the GPU"
                    self.waves.append(WaveRecord(wid, kind, w, len(reqs), est, tuples, t0, t1, held,
                                                 int(st.kernel_launches)))
                    total_held = sum(rr.prog.stats().device_bytes for rr in self._runners[w].values())
                    if total_held > self.budget / self.slots:
                        for rr in self._runners[w].values():
                            rr.prog.release()
                        total_held = 0
                    self._used[w] = float(total_held)
                    self._busy[w] = False
                    self.completed.extend(reqs)
                    current = None
                    self._cv.notify_all()
        except BaseException as e:  # surface worker failures to drain()
            with self._cv:
                self._errors.append(e)
                if current is not None:
                    self.failed_waves.append(current)
                self._cv.notify_all()

    def _retry_alone(self, w: int, runner: Runner, reqs):
        """A wave ran out of device memory (its estimate fell short): hold new
        admissions, wait for the other workers' waves, free every program's
        buffers, and rerun the wave alone -- split in halves while it still
        does not fit.  A request that does not fit alone gets no result."""
        with self._cv:
            self.oom_retries += 1
            self._busy[w] = False          # idle while waiting: another retrying worker may go first
            self._cv.notify_all()
            while self._exclusive is not None:
                self._cv.wait(0.05)
            self._exclusive = w
            self._busy[w] = True
            while any(self._busy[i] for i in range(self.slots) if i != w):
                self._cv.wait(0.05)
            self._release_idle(w)
        try:
            return self._run_split(w, runner, reqs)
        finally:
            if self.program_cap:
                runner.prog.set_memory_cap(self.program_cap)
            with self._cv:
                self._exclusive = None
                self._cv.notify_all()

    def _run_split(self, w: int, runner: Runner, reqs):
        for rr in self._runners[w].values():
            rr.prog.release()
        if self.program_cap:
            runner.prog.set_memory_cap(int(self.budget))
        try:
            return runner.run_wave([r.rows for r in reqs])
        except RAError as e:
            if e.status != E_OOM:
                raise
            if len(reqs) == 1:
                runner.prog.release()
                return [None]
            h = len(reqs) // 2
            return self._run_split(w, runner, reqs[:h]) + self._run_split(w, runner, reqs[h:])

    @staticmethod
    def _output(kind: str) -> str:
        return "T" if kind == "tc" else "SG"


# ---------------------------------------------------------------------- workloads


def request_mix(count: int, seed: int, tc_share: float = 0.8, large_share: float = 0.02,
                large_n: int = 1 << 18, large_degree: float = 0.95, n_hi: int = 16384,
                processes: int = 0) -> list[Request]:
    """The served mix: ``tc`` requests on ER graphs sized as the batched mix
    (n log-uniform in [64, n_hi = 16384], mean out-degree uniform in [0.8, 2.0]),
    ``sg`` requests on random trees of n log-uniform in [64, n_hi], and a
    share of large ``tc`` requests (ER, n = 2^18, mean out-degree 0.95).
    ``processes`` > 1 generates the graphs in a spawned process pool."""
    from . import datagen
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = datagen.batched_sizes(count, seed, n_hi=n_hi)
    kinds, specs = [], []
    for n, m, s in sizes:
        u = rng.uniform()
        if u < large_share:
            kinds.append("tc")
            specs.append(("er", large_n, round(large_degree * large_n), s))
        elif u < large_share + (1.0 - tc_share):
            kinds.append("sg")
            specs.append(("tree", n, s))
        else:
            kinds.append("tc")
            specs.append(("er", n, m, s))
    rows = datagen.generate_many(specs, processes)
    return [Request(i, k, r) for i, (k, r) in enumerate(zip(kinds, rows))]


def poisson_arrivals(count: int, rate: float, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def run_stream(server: Server, reqs: list[Request], arrivals: np.ndarray, timeout: float = 900.0) -> dict:
    """Submit ``reqs`` open-loop at ``arrivals`` (seconds) and wait for all of them."""
    for r, a in zip(reqs, arrivals):
        r.arrival = float(a)
        if not r.est_tuples:
            r.est_tuples = estimate_tuples(r.kind, r.rows)
        if not r.span:
            r.span = value_span(r.rows)
    base_done = len(server.completed)
    t0 = time.perf_counter()
    for r in reqs:
        delay = t0 + r.arrival - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        server.submit(r)
    server.drain(base_done + len(reqs), timeout)
    t1 = max(r.done for r in reqs)
    lat = np.array([r.latency for r in reqs]) * 1e3
    return {"requests": len(reqs), "offered_rate": len(reqs) / max(arrivals[-1], 1e-9),
            "seconds": t1 - t0, "instances_per_s": len(reqs) / (t1 - t0),
            "p50_ms": float(np.percentile(lat, 50)), "p95_ms": float(np.percentile(lat, 95)),
            "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(lat.max()),
            "mean_wave_size": float(np.mean([w.size for w in server.waves])) if server.waves else 0.0}
