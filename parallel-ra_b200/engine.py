"""ctypes binding of the B200 engine's C ABI (include/ra_engine.h).

``Program`` exposes the builder methods used by ``programs.py`` (relation /
load_rows / scc / add_relation / join / copy / depend) plus execute, history,
counts and dumps.  Every call goes to ``libra_b200.so``; there is no host
fallback: without the library or a GPU the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# RA_ENGINE_LIB: path of another build of the engine library (e.g. a tuning variant)
LIB_PATH = os.environ.get("RA_ENGINE_LIB") or os.path.join(HERE, "libra_b200.so")

# autotuner output (autotune.py); RA_TUNING_FILE names another file, or "none"
TUNING_PATH = os.path.join(HERE, "tuning.json")

DELTA, FULL = 0, 1
COPY, ACOPY, COPY_FILTER = 0, 1, 2
IDS_EMISSION, IDS_REFERENCE = 0, 1
# status codes of include/ra_engine.h
E_BADARG, E_IO, E_OOM, E_CUDA, E_UNSUPPORTED, E_TIMEOUT, E_STATE = 1, 2, 3, 4, 5, 6, 7

# every entry point declared in include/ra_engine.h
EXPORTS = (
    "ra_program_create", "ra_program_destroy", "ra_program_set_stream", "ra_program_set_batch_size",
    "ra_program_set_id_order", "ra_program_set_launch_timing", "ra_program_set_evaluators",
    "ra_relation_create", "ra_relation_load_rows", "ra_relation_load_rows_device", "ra_relation_load_file",
    "ra_scc_create", "ra_scc_add_relation", "ra_scc_add_join", "ra_scc_add_copy", "ra_scc_depend",
    "ra_program_execute", "ra_program_run_next_scc", "ra_program_reset", "ra_program_history", "ra_program_stats", "ra_program_iteration_times",
    "ra_relation_counts", "ra_relation_dump_full", "ra_rows_distinct_noalloc", "ra_status_string", "ra_last_error",
    "ra_program_set_instances", "ra_program_instance_history", "ra_relation_instance_summary",
    "ra_program_get_tuning", "ra_program_set_tuning", "ra_program_release",
    "ra_program_set_checkpoint", "ra_program_set_restart", "ra_program_set_memory_cap",
    "ra_selftest_bounded_wait", "ra_calibrate_random_access",
)


class RAError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint64), ("join_candidates", C.c_uint64), ("new_tuples", C.c_uint64),
        ("kernel_launches", C.c_uint64), ("fixpoint_ms", C.c_double), ("dedup_ms", C.c_double),
        ("dedup_launches", C.c_uint64), ("dedup_bytes", C.c_uint64), ("value_bits", C.c_uint32),
        ("reserved", C.c_uint32), ("phase_ms", C.c_double * 6), ("graph_builds", C.c_uint64),
        ("graph_build_ms", C.c_double), ("regrows", C.c_uint64), ("device_bytes", C.c_uint64),
        ("device_bytes_peak", C.c_uint64), ("dense_sccs", C.c_uint64), ("dense_search_ms", C.c_double),
        ("dense_emit_ms", C.c_double), ("bitmap_relations", C.c_uint64),
        ("persistent_launches", C.c_uint64), ("reach_sccs", C.c_uint64), ("reach_levels", C.c_uint64),
        ("reach_ms", C.c_double), ("reach_phase_ms", C.c_double * 4), ("sliced_iterations", C.c_uint64),
        ("sliced_passes", C.c_uint64), ("heavy_items", C.c_uint64), ("tail_iterations", C.c_uint64),
    ]
    PHASES = ("join_scan", "plan", "expand_claim", "select", "sort", "iter_end")


class Tuning(C.Structure):
    """ra_tuning: hash load factor, growth factors and kernel grid shapes of a program."""
    _fields_ = [
        ("seen_load_max", C.c_double), ("seen_grow", C.c_double), ("log_growth", C.c_double),
        ("join_blocks_per_sm", C.c_uint32), ("select_blocks_per_sm", C.c_uint32), ("dense_max_bytes", C.c_double),
    ]
    FIELDS = ("seen_load_max", "seen_grow", "log_growth", "join_blocks_per_sm", "select_blocks_per_sm",
              "dense_max_bytes")

    def as_dict(self):
        return {k: getattr(self, k) for k in self.FIELDS}


_lib = None


def lib():
    """Load libra_b200.so (built by build.py); raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run parallel-ra_b200/build.py (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        u64p = C.POINTER(C.c_uint64)
        i32p = C.POINTER(C.c_int)
        L.ra_program_create.argtypes = [C.c_int, C.POINTER(P)]
        L.ra_program_destroy.argtypes = [P]
        L.ra_program_set_stream.argtypes = [P, P]
        L.ra_program_set_batch_size.argtypes = [P, C.c_uint32]
        L.ra_program_set_id_order.argtypes = [P, C.c_int]
        L.ra_program_set_launch_timing.argtypes = [P, C.c_int]
        L.ra_program_set_evaluators.argtypes = [P, C.c_int, C.c_int]
        L.ra_relation_create.argtypes = [P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_char_p, C.c_int, i32p]
        L.ra_relation_load_rows.argtypes = [P, C.c_int, u64p, C.c_uint64]
        L.ra_relation_load_rows_device.argtypes = [P, C.c_int, C.c_void_p, C.c_uint64]
        L.ra_relation_load_file.argtypes = [P, C.c_int, C.c_char_p]
        L.ra_scc_create.argtypes = [P, C.c_int, C.c_int, i32p]
        L.ra_scc_add_relation.argtypes = [P, C.c_int, C.c_int, C.c_int]
        L.ra_scc_add_join.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, i32p, C.c_int]
        L.ra_scc_add_copy.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, i32p, C.c_int, C.c_int]
        L.ra_scc_depend.argtypes = [P, C.c_int, C.c_int]
        L.ra_program_execute.argtypes = [P]
        L.ra_program_run_next_scc.argtypes = [P, i32p]
        L.ra_program_reset.argtypes = [P]
        L.ra_program_release.argtypes = [P]
        L.ra_program_set_checkpoint.argtypes = [P, C.c_char_p, C.c_uint32, C.c_int]
        L.ra_program_set_restart.argtypes = [P, C.c_char_p, C.c_int]
        L.ra_program_set_memory_cap.argtypes = [P, C.c_uint64]
        L.ra_selftest_bounded_wait.argtypes = [C.c_int, C.c_uint64]
        L.ra_calibrate_random_access.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.POINTER(C.c_double)]
        L.ra_program_history.argtypes = [P, u64p, C.c_uint64, u64p]
        L.ra_program_stats.argtypes = [P, C.POINTER(Stats)]
        L.ra_program_iteration_times.argtypes = [P, C.POINTER(C.c_double), C.c_uint64, u64p]
        L.ra_relation_counts.argtypes = [P, C.c_int, u64p, u64p]
        L.ra_relation_dump_full.argtypes = [P, C.c_int, u64p, C.c_uint64, u64p]
        L.ra_program_set_instances.argtypes = [P, u64p, C.c_uint32]
        L.ra_program_get_tuning.argtypes = [P, C.POINTER(Tuning)]
        L.ra_program_set_tuning.argtypes = [P, C.POINTER(Tuning)]
        L.ra_program_instance_history.argtypes = [P, u64p, C.c_uint64, u64p]
        L.ra_relation_instance_summary.argtypes = [P, C.c_int, u64p, u64p]
        L.ra_rows_distinct_noalloc.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ra_status_string.argtypes = [C.c_int]
        L.ra_status_string.restype = C.c_char_p
        L.ra_last_error.argtypes = [P]
        L.ra_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def tuning_file() -> dict | None:
    """The autotuner's saved result, if any (see autotune.py)."""
    path = os.environ.get("RA_TUNING_FILE") or TUNING_PATH
    if path == "none" or not os.path.exists(path):
        return None
    import json
    with open(path) as f:
        return json.load(f)


def _u64(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


class Program:
    """One Datalog program on one GPU (an ``ra_program``)."""

    def __init__(self, device: int = 0, id_order: int | None = None):
        self._L = lib()
        h = C.c_void_p()
        st = self._L.ra_program_create(device, C.byref(h))
        if st != 0:
            raise RAError(st, f"ra_program_create(device={device}): {self._L.ra_status_string(st).decode()}")
        self._p = h
        self._arity = {}
        self._n_inst = 0
        tuned = tuning_file()
        if tuned:
            self.set_tuning(**tuned["tuning"])
        if id_order is not None:
            self.set_id_order(id_order)

    def _ck(self, st, what):
        if st != 0:
            raise RAError(st, f"{what}: {self._L.ra_status_string(st).decode()}: "
                              f"{self._L.ra_last_error(self._p).decode()}")

    def close(self):
        if getattr(self, "_p", None):
            self._L.ra_program_destroy(self._p)
            self._p = None

    def __del__(self):
        self.close()

    @property
    def handle(self):
        return self._p

    def set_stream(self, stream_ptr: int):
        self._ck(self._L.ra_program_set_stream(self._p, C.c_void_p(stream_ptr)), "set_stream")

    def set_id_order(self, mode: int):
        """IDS_EMISSION (default) or IDS_REFERENCE (single-rank reference numbering)."""
        self._ck(self._L.ra_program_set_id_order(self._p, mode), "set_id_order")

    def set_launch_timing(self, on: bool):
        """Per-launch CUDA events on every iteration kernel (no CUDA graph while on)."""
        self._ck(self._L.ra_program_set_launch_timing(self._p, int(bool(on))), "set_launch_timing")

    def set_evaluators(self, reach: bool = True, persistent: bool = False):
        """reach: closure-shaped SCCs by composing reachable sets; persistent: other
        device-driven SCCs as one cooperative launch (results are the same either way)."""
        self._ck(self._L.ra_program_set_evaluators(self._p, int(bool(reach)), int(bool(persistent))),
                 "set_evaluators")

    def set_batch_size(self, n: int):
        self._ck(self._L.ra_program_set_batch_size(self._p, n), "set_batch_size")

    def relation(self, jcc, arity, tag, name, version=FULL):
        out = C.c_int()
        self._ck(self._L.ra_relation_create(self._p, jcc, arity, tag, name.encode(), version, C.byref(out)),
                 "relation")
        self._arity[out.value] = arity
        return out.value

    def load_rows(self, rel, rows: np.ndarray):
        rows = np.ascontiguousarray(rows, dtype=np.uint64)
        self._ck(self._L.ra_relation_load_rows(self._p, rel, _u64(rows), rows.shape[0]), "load_rows")

    def load_rows_device(self, rel, dev_ptr: int, nrows: int):
        self._ck(self._L.ra_relation_load_rows_device(self._p, rel, C.c_void_p(dev_ptr), nrows), "load_rows_device")

    def load_file(self, rel, path: str):
        self._ck(self._L.ra_relation_load_file(self._p, rel, path.encode()), "load_file")

    def scc(self, fixpoint, scc_id):
        out = C.c_int()
        self._ck(self._L.ra_scc_create(self._p, int(bool(fixpoint)), scc_id, C.byref(out)), "scc")
        return out.value

    def add_relation(self, scc, rel, init_status):
        self._ck(self._L.ra_scc_add_relation(self._p, scc, rel, int(bool(init_status))), "add_relation")

    def join(self, scc, out, in0, ver0, in1, ver1, proj):
        arr = (C.c_int * len(proj))(*proj)
        self._ck(self._L.ra_scc_add_join(self._p, scc, out, in0, ver0, in1, ver1, arr, len(proj)), "join")

    def copy(self, scc, out, src, ver, proj, kind=COPY, pred=0):
        arr = (C.c_int * len(proj))(*proj)
        self._ck(self._L.ra_scc_add_copy(self._p, scc, kind, out, src, ver, arr, len(proj), pred), "copy")

    def depend(self, src_scc, dst_scc):
        self._ck(self._L.ra_scc_depend(self._p, src_scc, dst_scc), "depend")

    def execute(self, batch_size: int | None = None):
        if batch_size is not None:
            self.set_batch_size(batch_size)
        self._ck(self._L.ra_program_execute(self._p), "execute")

    def set_checkpoint(self, output_dir: str, every_batches: int, separate_files: bool = False):
        """Write the reference's checkpoint dumps every ``every_batches`` batches (0: off)."""
        self._ck(self._L.ra_program_set_checkpoint(self._p, output_dir.encode(), every_batches,
                                                   1 if separate_files else 0), "set_checkpoint")

    def set_restart(self, dump_dir: str | None, separate_files: bool = False):
        """Resume from a checkpoint dump directory (None: no restart)."""
        self._ck(self._L.ra_program_set_restart(self._p, (dump_dir or "").encode(), 1 if separate_files else 0),
                 "set_restart")

    def set_memory_cap(self, nbytes: int):
        """Most device bytes the program may hold (0: no cap); beyond it a run fails with E_OOM."""
        self._ck(self._L.ra_program_set_memory_cap(self._p, int(nbytes)), "set_memory_cap")

    def release(self):
        """Free the device buffers kept between runs (ends the last run)."""
        self._ck(self._L.ra_program_release(self._p), "release")

    def reset(self):
        self._ck(self._L.ra_program_reset(self._p), "reset")

    def history(self):
        """[(scc_id, [(sum_delta, sum_full), ...]), ...] in execution order."""
        n = C.c_uint64()
        self._ck(self._L.ra_program_history(self._p, None, 0, C.byref(n)), "history")
        buf = np.zeros(max(n.value, 1), dtype=np.uint64)
        self._ck(self._L.ra_program_history(self._p, _u64(buf), n.value, C.byref(n)), "history")
        out, i = [], 0
        while i < n.value:
            sid, k = int(buf[i]), int(buf[i + 1])
            pairs = [(int(buf[i + 2 + 2 * j]), int(buf[i + 3 + 2 * j])) for j in range(k)]
            out.append((sid, pairs))
            i += 2 + 2 * k
        return out

    def stats(self) -> Stats:
        s = Stats()
        self._ck(self._L.ra_program_stats(self._p, C.byref(s)), "stats")
        return s

    def iteration_times_us(self):
        """Device time of each device-driven iteration of the last run (microseconds)."""
        n = C.c_uint64()
        self._ck(self._L.ra_program_iteration_times(self._p, None, 0, C.byref(n)), "iteration_times")
        buf = (C.c_double * max(n.value, 1))()
        self._ck(self._L.ra_program_iteration_times(self._p, buf, n.value, C.byref(n)), "iteration_times")
        return list(buf)[:n.value]

    def counts(self, rel):
        f, d = C.c_uint64(), C.c_uint64()
        self._ck(self._L.ra_relation_counts(self._p, rel, C.byref(f), C.byref(d)), "counts")
        return f.value, d.value

    def full_count(self, rel):
        return self.counts(rel)[0]

    def dump_full(self, rel):
        """Full relation rows (data columns + id) in lexicographic order."""
        n = self.full_count(rel)
        w = self._arity[rel] + 1
        buf = np.zeros((max(n, 1), w), dtype=np.uint64)
        got = C.c_uint64()
        self._ck(self._L.ra_relation_dump_full(self._p, rel, _u64(buf), n, C.byref(got)), "dump_full")
        return buf[:got.value]

    def set_instances(self, value_base):
        """Declare the instances of a batched run (value_base[i]: first value of instance i)."""
        vb = np.ascontiguousarray(value_base, dtype=np.uint64)
        self._n_inst = int(vb.size)
        self._ck(self._L.ra_program_set_instances(self._p, _u64(vb) if vb.size else None, vb.size),
                 "set_instances")

    def instance_history(self) -> np.ndarray:
        """New tuples per (iteration, instance) of the last run, shape (iterations, instances)."""
        n = C.c_uint64()
        self._ck(self._L.ra_program_instance_history(self._p, None, 0, C.byref(n)), "instance_history")
        buf = np.zeros((max(n.value, 1), self._n_inst), dtype=np.uint64)
        self._ck(self._L.ra_program_instance_history(self._p, _u64(buf), n.value, C.byref(n)), "instance_history")
        return buf[:n.value]

    def instance_summary(self, rel):
        """Per-instance (row count, data digest) of a relation's full version, as two arrays."""
        m = max(self._n_inst, 1)
        counts = np.zeros(m, dtype=np.uint64)
        digests = np.zeros(m, dtype=np.uint64)
        self._ck(self._L.ra_relation_instance_summary(self._p, rel, _u64(counts), _u64(digests)),
                 "instance_summary")
        return counts, digests

    def get_tuning(self) -> dict:
        t = Tuning()
        self._ck(self._L.ra_program_get_tuning(self._p, C.byref(t)), "get_tuning")
        return t.as_dict()

    def set_tuning(self, **kw):
        """Change some tuning fields (see ra_tuning in include/ra_engine.h); others keep their values."""
        t = Tuning()
        self._ck(self._L.ra_program_get_tuning(self._p, C.byref(t)), "get_tuning")
        for k, v in kw.items():
            if k not in Tuning.FIELDS:
                raise KeyError(k)
            setattr(t, k, v)
        self._ck(self._L.ra_program_set_tuning(self._p, C.byref(t)), "set_tuning")


def selftest_bounded_wait(device: int = 0, max_polls: int = 1 << 16) -> int:
    """Status of the engine's bounded-wait self-test (E_TIMEOUT when the wait gave up as designed)."""
    return lib().ra_selftest_bounded_wait(device, max_polls)


def calibrate_random_access(device: int = 0, slots: int = 177 << 20, ops: int = 64 << 20) -> dict:
    """This GPU's random 16-byte CAS and 8-byte load rates (operations/s) on a table
    of `slots` 16-byte slots: the ceiling of the seen-set claims."""
    out = (C.c_double * 2)()
    st = lib().ra_calibrate_random_access(device, slots, ops, out)
    if st != 0:
        raise RAError(st, f"ra_calibrate_random_access: {lib().ra_status_string(st).decode()}")
    return {"cas16_per_s": out[0], "load8_per_s": out[1], "table_bytes": 16 * slots}

