#!/usr/bin/env python
"""Benchmark of parallel-RA's semi-naive fixed point on B200.

Workload (default ``tc-er22``): the transitive-closure program of the
reference (tests/transitive_closure.cpp) on a seeded directed Erdos-Renyi
graph with 2^22 nodes and m = 3,984,589 distinct edges (mean out-degree
0.95, no self-loops), ids in the reference's binary relation layout.

One step = one LIE::execute of the whole program (copy SCC + join SCC to its
fixed point) on relations already resident in HBM; the metric is final
|TC| tuples per second of device time.  ``e2e`` measures the same through
the public C ABI from pinned host rows: upload, packing, fixed point and the
read-back of the per-relation counts and the per-iteration history.

``--impl reference`` times the reference's own CPU code (oracle/_ref, the
unchanged parallel-RA sources on a single-rank MPI stand-in).

Launch: ``python bench.py [--gpus N --steps K --warmup W]``; for N > 1 under
torchrun, each rank runs its own seeded instance (instance-parallel replicas).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TC tuples/s"
METRIC_FAMILY = "TC tuples/s + HBM GB/s on 1 B200; batched vs serial instances/s; p99 ms"
WORKLOADS = {
    # name: (program, graph generator, generator arguments)
    "tc-er22": ("tc", "er", (1 << 22, 3984589, 2)),
    "tc-er20": ("tc", "er", (1 << 20, 996147, 2)),    # same family at 1/4 scale (profiling case)
    "tc-er2000": ("tc", "er", (2000, 3000, 1)),
    "sg-tree15": ("sg", "tree", (1 << 15, 3)),         # same generation on a random tree of 2^15 nodes
    # the largest instance class of the batched mix: a dense closure (dense row-closure evaluator)
    "tc-er16384d2": ("tc", "er", (16384, 32768, 7)),
}
# the reference's generated analyses, as program descriptions + relation files
# (tests/golden/<name>/, written from the reference's tests/<name>.cpp): wide tuples
DESCRIBED = {"worstcase-110-terms-4-m": "0-CFA-style analysis of a generated 110-term program "
                                        "(60 relations, arity <= 13, 19 SCCs, batch size 10)",
             "cfa-4-4-64": "k-CFA analysis (37 relations, arity <= 23, joins on 0..16 columns)"}
OUTPUT = {"tc": "T", "sg": "SG"}
INPUT = {"tc": "G", "sg": "edge"}
# bounded CPU samples of the same graph families (the cpu_baseline of our arm, and the
# reference arm of workloads in REFERENCE_SAMPLED)
CPU_SAMPLES = {"tc": ("er", (1 << 17, round(0.95 * (1 << 17)), 2)), "sg": ("tree", (1 << 12, 3))}
# the reference's same generation on the 2^15-node tree holds 5.5e8 tuples in its B-tree
# tries: a 73.7 GB peak (measured when its golden was generated, 694 s of fixpoint on one
# core); on a host with less free memory than the figure below, its reference arm
# runs the 2^12-node sample instead
REFERENCE_SAMPLED = {"sg-tree15": 96 << 30}
REFERENCE_ARM_SECONDS = 600.0
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (read + write) per algorithmic byte of join_fused_kernel, from the
# ncu capture in profiles/join_fused_kernel_tc-er20.md (1.93 / 1.93 / 1.95 over
# three launches of the same graph family at 1/4 scale); bench's `traffic` is
# this ratio times the algorithmic bytes of an average tc-er22 launch.
TRAFFIC_PER_ALGO_BYTE = 1.94


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def workload_rows(gen, params):
    import parallel_ra_b200 as P
    if gen == "er":
        return P.datagen.with_row_ids(P.datagen.erdos_renyi(*params))
    return P.datagen.with_row_ids(P.datagen.random_tree(*params))


def reference_sample_run(kind):
    """The reference's CPU code on the bounded sample of a program's graph family."""
    gen, params = CPU_SAMPLES[kind]
    return reference_rows_run(workload_rows(gen, params), kind)


def reference_rows_run(rows, kind="tc"):
    """Program ``kind`` on ``rows`` by the reference's CPU code; returns (output tuples, fixpoint seconds, kind)."""
    import parallel_ra_b200 as P
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if os.path.exists(drv):
        with tempfile.TemporaryDirectory() as tmp:
            edge, empty, out = (os.path.join(tmp, x) for x in ("edge", "empty", "out"))
            P.datagen.write_relation(edge, rows)
            P.datagen.write_empty_relation(empty)
            subprocess.run([drv, kind, edge, empty, out], check=True, stdout=subprocess.DEVNULL,
                           env=dict(os.environ, RA_REF_NODUMP="1"))
            secs = float(open(os.path.join(out, "time.txt")).read())
            tc = next(int(l.split()[2]) for l in open(os.path.join(out, "sizes.txt"))
                      if l.split()[0] == OUTPUT[kind])
        return tc, secs, "reference"
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    p = O.OracleProgram()
    rels = P.programs.PROGRAMS[kind](p, rows)
    p.execute(1)
    return p.full_count(rels[OUTPUT[kind]]), p.fixpoint_seconds(), "port"


def cpu_sample_desc(kind="tc"):
    gen, params = CPU_SAMPLES[kind]
    if gen == "er":
        n, m, s = params
        return (f"TC on ER n={n} m={m} seed={s} (same family as the workload, mean out-degree 0.95), "
                f"fixpoint time only")
    n, s = params
    return f"SG on a random tree of n={n} nodes seed={s} (same family as the workload), fixpoint time only"


def accumulate_dense(acc, st):
    """Add a run's dense-evaluator figures (filled with per-launch timing) to ``acc``."""
    if st.dense_sccs:
        acc["search_ms"] += st.dense_search_ms
        acc["emit_ms"] += st.dense_emit_ms
        acc["sccs"] += st.dense_sccs
        acc["new_tuples"] += st.new_tuples
        acc["candidates"] += st.join_candidates


def dense_roofline(d, peak, peak_kind):
    """Roofline of the dense row-closure evaluator's kernels.  The emission kernel is
    HBM-bound: 16 B written per new tuple (key + id).  The row searches run in shared
    memory against an L2-resident adjacency; their bound is SM issue, not DRAM, so they
    are reported with their time share and edge rate beside the HBM roofline."""
    achieved = 16.0 * d["new_tuples"] / (d["emit_ms"] / 1e3) / 1e9 if d["emit_ms"] else 0.0
    tot = d["search_ms"] + d["emit_ms"]
    return {"kernel": "dense_emit_kernel", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
            "bytes_model": "16 B written per new tuple (key + id)",
            "share_of_dense_time": d["emit_ms"] / tot if tot else None,
            "dense_search": {"kernels": "dense_closure_kernel / dense_closure_warp_kernel", "ms": d["search_ms"],
                             "share_of_dense_time": d["search_ms"] / tot if tot else None,
                             "edges_per_s": d["candidates"] / (d["search_ms"] / 1e3) if d["search_ms"] else None,
                             "bound": "SM issue: shared-memory bit sets and atomics, adjacency L2-resident "
                                      "(ncu: sm__throughput ~73%, DRAM idle)"}}


def reduce_ranks(total_ms, count, device):
    """Whole-job figures of N independent replicas: the slowest rank's device time
    (MAX) and the units all ranks processed (SUM).  One rank: unchanged."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(total_ms), int(count)
    if dist.get_backend() == "gloo":
        device = "cpu"
    t = torch.tensor([float(total_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(count)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), int(c.item())


def metric_of(kind):
    return f"{OUTPUT[kind]} tuples/s" if kind == "sg" else METRIC


def host_free_bytes() -> int:
    """Host memory available to a new process (MemAvailable), 0 if unknown."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def run_reference_arm(args, rank, world):
    if rank != 0:
        return None
    if args.workload in DESCRIBED:
        vals = [described_reference_run(args.workload) for _ in range(max(1, min(args.steps, 2)))]
        facts, secs = vals[0][0], sum(v[1] for v in vals) / len(vals)
        sample = f"the whole program on the reference library, {len(vals)} run(s)"
        return {"impl": "reference", "metric": "facts/s", "value": facts / secs, "unit": "facts/s",
                "n_gpus": args.gpus, "steps": len(vals), "warmup": 0, "ms_per_step": 1e3 * secs,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
                "data": "the reference's own input relations", "config": {"workload": args.workload,
                                                                           "metric_family": METRIC_FAMILY},
                "cpu_baseline": {"value": facts / secs, "unit": "facts/s", "cores": 1, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": facts / secs, "unit": "facts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "served":
        # the reference serves one request at a time: its throughput on a bounded sample of
        # the served mix (requests whose closure is estimated below 5e6 tuples), converted
        # to instances/s over the whole mix by the mix's estimated tuples
        from parallel_ra_b200.batch import estimate_tuples
        from parallel_ra_b200.serve import request_mix
        reqs = request_mix(SERVED_COUNT, SERVED_SEED, processes=gen_processes())
        est = [estimate_tuples(r.kind, r.rows) for r in reqs]
        rng = np.random.default_rng(7)
        pool = [int(i) for i in rng.permutation(len(reqs)) if est[int(i)] < 5e6][:BATCH_CPU_SAMPLE]
        tup = secs = 0.0
        kind = "port"
        for i in pool:
            t, sec, kind = reference_rows_run(reqs[i].rows, reqs[i].kind)
            tup += t
            secs += sec
        value = len(reqs) / (sum(est) / (tup / secs))
        sample = (f"{len(pool)} random requests of the mix with estimated closure < 5e6 tuples ({int(tup)} "
                  f"tuples, {secs:.1f} s fixpoint time); instances/s = requests / (mix tuples / sample tuples/s)")
        return {"impl": "reference", "metric": "served instances/s", "value": value, "unit": "instances/s",
                "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * len(reqs) / value,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": {"workload": "served", "requests": SERVED_COUNT, "metric_family": METRIC_FAMILY},
                "cpu_baseline": {"value": value, "unit": "instances/s", "cores": 1, "kind": kind, "sample": sample},
                "e2e": {"value": value, "unit": "instances/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "batched":
        from parallel_ra_b200.batch import estimate_tuples
        insts = batched_instances(BATCH_COUNT, BATCH_SEED)
        total = sum(estimate_tuples("tc", r) for r in insts)
        cb = batched_cpu_baseline(insts, total)
        cb["sample"] += "; batch tuples from the closure-size estimate"
        per_step = BATCH_COUNT / cb["value"]
        return {"impl": "reference", "metric": "batched TC instances/s", "value": cb["value"],
                "unit": "instances/s", "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * per_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
                "data": "synthetic", "config": {"workload": "batched", "instances": BATCH_COUNT,
                                                "metric_family": METRIC_FAMILY},
                "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "instances/s", "h2d_bytes_per_step": 0,
                                            "d2h_bytes_per_step": 0}}
    prog_kind, gen, params = WORKLOADS[args.workload]
    if args.workload in REFERENCE_SAMPLED and host_free_bytes() < REFERENCE_SAMPLED[args.workload]:
        # the reference needs more host memory than this host has free (see REFERENCE_SAMPLED)
        rows, desc, same = None, cpu_sample_desc(prog_kind), False
    else:
        rows = workload_rows(gen, params)
        desc = (f"the workload's own input ({args.workload}: {gen} {list(params)}, {rows.shape[0]} rows), "
                f"fixpoint time only")
        same = True
    # every step is a whole run of the reference (minutes at 2^22 nodes on one core): steps
    # are taken while the arm's time stays within REFERENCE_ARM_SECONDS, at least one
    vals = []
    t_start = time.time()
    while len(vals) < args.steps:
        tc, secs, kind = reference_rows_run(rows, prog_kind) if rows is not None else reference_sample_run(prog_kind)
        vals.append((tc, secs))
        if time.time() - t_start > REFERENCE_ARM_SECONDS * len(vals) / (len(vals) + 1):
            break
    tot_tc = sum(v[0] for v in vals)
    tot_s = sum(v[1] for v in vals)
    value = tot_tc / tot_s
    line = {
        "impl": "reference", "metric": metric_of(prog_kind), "value": value, "unit": "tuples/s", "n_gpus": args.gpus,
        "steps": len(vals), "warmup": 0, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": 1e3 * tot_s / len(vals), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": args.workload, "sample": desc, "same_config": same, "output_tuples": vals[0][0],
                   "steps_note": "each step is one whole run of the reference on one core; no warm-up (CPU "
                                 "code, nothing to compile or cache across runs)",
                   "metric_family": METRIC_FAMILY},
        "cpu_baseline": {"value": value, "unit": "tuples/s", "cores": 1, "kind": kind, "sample": desc},
        "e2e": {"value": value, "unit": "tuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def run_ours(args, rank, world, local_rank):
    import torch
    import parallel_ra_b200 as P

    dev = local_rank % max(1, torch.cuda.device_count())
    torch.cuda.set_device(dev)
    prog_kind, gen, params = WORKLOADS[args.workload]
    partitioned = world > 1 and prog_kind == "tc" and gen == "er"
    if partitioned:
        # one instance N times the size, T partitioned over the ranks by source (partition.py):
        # every rank generates the same graph, keeps G whole and seeds T with the edges it owns
        n, m, seed = params
        params = (n * world, m * world, seed)
    else:
        params = params[:-1] + (params[-1] + 1000 * rank,)     # each rank: its own independent instance
    rows = workload_rows(gen, params)
    stream = torch.cuda.Stream()
    prog = P.Program(dev)
    prog.set_stream(stream.cuda_stream)
    if partitioned:
        rels = P.partition.build_tc_partitioned(prog, rows, rank, world)
        own = P.partition.owner(rows[:, 0], world) == rank
        inputs = {"G": rows, "G_own": np.ascontiguousarray(rows[own]), "T": np.empty((0, 3), dtype=np.uint64)}
    else:
        rels = P.programs.PROGRAMS[prog_kind](prog, rows)
        inputs = {name: (rows if name == INPUT[prog_kind] else np.empty((0, 3), dtype=np.uint64)) for name in rels}
    out_rel = rels[OUTPUT[prog_kind]]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=f"cuda:{dev}")

    for _ in range(args.warmup):
        prog.execute(1)
    tc = prog.full_count(out_rel)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches = 0
    torch.cuda.synchronize()
    profile_range = bool(os.environ.get("RA_PROFILE_TIMED"))   # ncu --profile-from-start off
    if profile_range:
        torch.cuda.profiler.start()
    with ClockSampler(local_rank) as clocks:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()                  # L2 flush between steps, outside the timed events
            starts[i].record(stream)
            prog.execute(1)
            ends[i].record(stream)
            launches += prog.stats().kernel_launches
        torch.cuda.synchronize()
    if profile_range:
        torch.cuda.profiler.stop()
    if world > 1:
        torch.distributed.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms, tc_all = reduce_ranks(sum(step_ms), tc, f"cuda:{dev}")
    value = tc_all * args.steps / (total_ms / 1e3)
    st = prog.stats()
    iterations = int(st.iterations)
    if partitioned:
        # the single-instance history from every rank's (one exchange, after the timing)
        gh = P.partition.global_history(prog.history())
        iterations = sum(len(h) for _, h in gh)

    # dominant kernel (fused join count, scan, expansion + first-occurrence claim): per-launch
    # CUDA events on the engine's stream, in an instrumented pass over the same
    # program (the timed steps run as one CUDA graph, whose nodes events cannot split)
    prog.set_launch_timing(True)
    dedup_ms = dedup_bytes = dedup_launches = 0
    phase = [0.0] * 6
    dense = {"search_ms": 0.0, "emit_ms": 0.0, "sccs": 0, "new_tuples": 0, "candidates": 0}
    for _ in range(max(1, min(args.steps, 3))):
        prog.execute(1)
        s2 = prog.stats()
        dedup_ms += s2.dedup_ms
        dedup_bytes += s2.dedup_bytes
        dedup_launches += s2.dedup_launches
        phase = [a + b for a, b in zip(phase, s2.phase_ms)]
        accumulate_dense(dense, s2)
    prog.set_launch_timing(False)

    # the same program with intern ids numbered exactly as the single-rank reference
    prog.set_id_order(P.engine.IDS_REFERENCE)
    ref_ms = []
    for _ in range(3):
        prog.execute(1)
        ref_ms.append(prog.stats().fixpoint_ms)
    prog.set_id_order(P.engine.IDS_EMISSION)

    # end to end through the C ABI from pinned host rows
    pinned_in = {name: torch.from_numpy(np.ascontiguousarray(r).view(np.int64)).pin_memory().numpy().view(np.uint64)
                 for name, r in inputs.items()}
    h2d_bytes = int(sum(r.nbytes for r in inputs.values()))

    def load_inputs():
        for name, r in pinned_in.items():
            prog.load_rows(rels[name], r)

    e2e_s = []
    d2h = 0
    for i in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        load_inputs()
        prog.execute(1)
        h = prog.history()
        f, _ = prog.counts(out_rel)
        e2e_s.append(time.perf_counter() - t0)
        d2h = 8 * (2 + sum(2 + 2 * len(x[1]) for x in h))
        assert f == tc
    e2e_ms, e2e_units = reduce_ranks(1e3 * statistics.mean(e2e_s), tc, f"cuda:{dev}")
    e2e = {"value": e2e_units / (e2e_ms / 1e3), "unit": "tuples/s", "h2d_bytes_per_step": h2d_bytes,
           "d2h_bytes_per_step": int(d2h)}
    # the same, for a caller that wants the derived relation itself: its rows (data columns
    # and intern ids, trie order) read back to host memory inside the timed region
    e2e_rows_s = []
    rows_d2h = 0
    for i in range(max(1, min(args.steps, 2))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        load_inputs()
        prog.execute(1)
        h = prog.history()
        out_rows = prog.dump_full(out_rel)
        e2e_rows_s.append(time.perf_counter() - t0)
        rows_d2h = int(out_rows.nbytes) + 8 * (2 + sum(2 + 2 * len(x[1]) for x in h))
        assert out_rows.shape[0] == tc
        del out_rows
    er_ms, er_units = reduce_ranks(1e3 * statistics.mean(e2e_rows_s), tc, f"cuda:{dev}")
    e2e_rows = {"value": er_units / (er_ms / 1e3), "unit": "tuples/s", "h2d_bytes_per_step": h2d_bytes,
                "d2h_bytes_per_step": rows_d2h,
                "note": "e2e plus ra_relation_dump_full of the output relation (sorted rows with ids) to host"}

    peak, peak_kind = load_peaks()
    achieved = (dedup_bytes / dedup_launches) / ((dedup_ms / dedup_launches) / 1e3) / 1e9 if dedup_launches else 0.0
    bitmap = st.bitmap_relations > 0
    roofline = dense_roofline(dense, peak, peak_kind) if dense["sccs"] else {"kernel": "join_fused_kernel", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": None if bitmap else TRAFFIC_PER_ALGO_BYTE * dedup_bytes / max(dedup_launches, 1),
                "traffic_note": ("not captured for the bitmap path" if bitmap else
                                 "ncu DRAM read+write per launch, measured on tc-er20 and scaled by units processed"),
                "launches": int(dedup_launches), "avg_launch_us": 1e3 * dedup_ms / max(dedup_launches, 1),
                "bytes_per_launch": dedup_bytes / max(dedup_launches, 1),
                "bytes_model": ("8 B per candidate (the inner key; the claim is a bit test and an atomicOr on a "
                                "bitmap word, mostly L2-resident) + 24 B per outer delta row" if bitmap else
                                "48 B per candidate (8 B inner key read, 8 B candidate write, 16 B seen-slot read "
                                "+ 16 B write) + 24 B per outer delta row (key, row offset, CSR start)")}
    if not dense["sccs"] and not bitmap and dedup_launches and world == 1:
        # the claims' own ceiling on this GPU: random 16-byte CAS on a table of the seen set's size
        cal = P.engine.calibrate_random_access(dev, slots=max(1 << 20, int(tc / 0.45)), ops=64 << 20)
        claims_per_s = st.join_candidates / (dedup_ms / max(1, min(args.steps, 3)) / 1e3) if dedup_ms else 0.0
        roofline["random_access_ceiling"] = {
            "cas16_per_s": cal["cas16_per_s"], "load8_per_s": cal["load8_per_s"], "table_bytes": cal["table_bytes"],
            "claims_per_s": claims_per_s, "claims_frac_of_cas16": claims_per_s / cal["cas16_per_s"],
            "note": "every candidate claims one 16-byte slot of a table far larger than L2; this GPU's rate "
                    "of such random read-modify-writes, measured here, bounds the join kernel below the "
                    "HBM copy roofline (linear probing adds ~1.3-2 CAS per candidate)"}

    if rank != 0:
        return None
    line = {
        "metric": metric_of(prog_kind), "value": value, "unit": "tuples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": args.workload, "program": prog_kind, "generator": gen, "generator_args": list(params),
                   "input_rows": int(rows.shape[0]), "output_tuples": tc_all, "iterations": iterations,
                   "join_candidates": int(st.join_candidates),
                   "value_bits": int(st.value_bits), "l2": "flushed (256 MiB write) before every timed step",
                   "id_order": "emission (default)",
                   "value_reference_ids": tc / (statistics.median(ref_ms) / 1e3),
                   "phase_ms_per_step": {k: v / max(1, min(args.steps, 3)) for k, v in
                                         zip(P.engine.Stats.PHASES, phase)},
                   "parallelism": (f"one instance of {world}x the size, T partitioned over {world} ranks by a hash of "
                                   f"its source column, G replicated; no exchange (partition.py)" if partitioned else
                                   f"{world} independent instance(s), one per GPU"),
                   "metric_family": METRIC_FAMILY},
        "clocks": clocks.summary(), "e2e": e2e, "e2e_with_rows": e2e_rows, "gpu_launches": int(launches),
        "roofline": roofline, "step_ms": step_ms,
    }
    if world == 1 and not args.no_cpu_baseline:
        ctc, csecs, kind = reference_sample_run(prog_kind)
        line["cpu_baseline"] = {"value": ctc / csecs, "unit": "tuples/s", "cores": 1, "kind": kind,
                                "sample": cpu_sample_desc(prog_kind)}
        golden = os.path.join(ROOT, "tests", "golden", GOLDEN_OF.get(args.workload, "") + ".json")
        if args.workload in GOLDEN_OF and os.path.exists(golden):
            g = json.load(open(golden))
            if "reference_fixpoint_seconds_1core" in g:
                line["cpu_baseline"]["same_input_reference_seconds"] = g["reference_fixpoint_seconds_1core"]
                line["cpu_baseline"]["same_input_note"] = (
                    "the reference's fixpoint time on this very input, one core, recorded when the golden "
                    "vectors were generated (tests/golden/make_golden.py); `bench.py --impl reference` "
                    "times it again on this box")
    if world == 1 and args.workload == "tc-er22" and not args.no_extras:
        # the other two patterns of the headline metric, bounded, in the same driver-run record
        line["config"]["batched"] = batched_summary(args, local_rank)
        line["config"]["served"] = served_summary(args, local_rank)
    return line


# the golden record of each workload's own input (reference run), when one exists
GOLDEN_OF = {"tc-er22": "er4194304_tc", "sg-tree15": "tree32768_sg", "tc-er2000": "er2000_tc"}


def batched_summary(args, local_rank):
    """The batched workload (8,192 TC instances against plain one-instance runs), one timed pass."""
    sub = argparse.Namespace(**vars(args))
    sub.steps, sub.warmup = 1, 1
    line = run_batched(sub, 0, 1, local_rank)
    return {"instances": line["config"]["instances"], "instances_per_s": line["value"],
            "e2e_instances_per_s": line["e2e"]["value"], "serial_instances_per_s": line["serial"]["value"],
            "batched_over_serial": line["value"] / line["serial"]["value"],
            "batched_e2e_over_serial": line["serial"]["batched_e2e_over_serial"],
            "bit_exact_mismatches": line["serial"]["bit_exact_mismatches"], "waves": line["config"]["waves"],
            "tuples_per_s": line["config"]["tuples_per_s"], "gpu_launches": line["gpu_launches"],
            "step": "one timed pass over the batch (union rows resident), serial = plain runs of a random "
                    f"sample of {BATCH_SERIAL_SAMPLE} instances from host rows, each checked bit-exact"}


def served_summary(args, local_rank):
    """The served workload at one arrival rate (the top of the sweep)."""
    sub = argparse.Namespace(**vars(args))
    sub.steps, sub.warmup = 1, 1
    line = run_served(sub, 0, 1, local_rank, rates=(max(SERVED_RATES),))
    pt = line["config"]["rates"][0]
    return {"rate_per_s": pt["rate"], "requests": line["config"]["requests"], "instances_per_s": line["value"],
            "p50_ms": pt["p50_ms"], "p95_ms": pt["p95_ms"], "p99_ms": pt["p99_ms"],
            "one_at_a_time_instances_per_s": line["one_at_a_time"]["value"],
            "served_over_one_at_a_time": line["value"] / line["one_at_a_time"]["value"],
            "bit_exact_checked": line["bit_exact"]["checked"], "bit_exact_mismatches": line["bit_exact"]["mismatches"],
            "oom_retries": line["admission"]["oom_retries"], "waves": pt["waves"]}


def described_paths(name):
    d = os.path.join(ROOT, "tests", "golden", name)
    return os.path.join(d, "program.txt"), os.path.join(d, "data")


def described_reference_run(name):
    """The reference library on the described program (oracle/_ref/ref_driver, one
    core): (total facts, fixpoint seconds = the sum of its execute_in_batches calls)."""
    import tempfile
    import parallel_ra_b200 as P
    prog, data = described_paths(name)
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    with tempfile.TemporaryDirectory() as work:
        empty = os.path.join(work, "empty")
        P.datagen.write_empty_relation(empty)
        out = os.path.join(work, "out")
        subprocess.run([drv, "file", prog, empty, out, data], check=True, stdout=subprocess.DEVNULL)
        facts = sum(int(ln.split()[2]) for ln in open(os.path.join(out, "sizes.txt")))
        secs = float(open(os.path.join(out, "time.txt")).read())
    return facts, secs


def run_described_ours(args, rank, world, local_rank):
    """A generated analysis on the wide-tuple path: facts/s = all relations' final
    tuples over the device time of one LIE::execute (relations resident in HBM)."""
    import torch
    import parallel_ra_b200 as P

    torch.cuda.set_device(local_rank)
    prog_path, data = described_paths(args.workload)
    stream = torch.cuda.Stream()
    prog = P.Program(local_rank)
    prog.set_stream(stream.cuda_stream)
    rels = P.programs.build_described(prog, prog_path, data)
    batch = rels.pop("__batch__")
    host_rows = {name: P.datagen.read_relation(os.path.join(data, f)) for name, f in
                 ((r["name"], r["file"]) for r in P.programs.read_description(prog_path)["relations"]) if f}
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=f"cuda:{local_rank}")
    for _ in range(args.warmup):
        prog.execute(batch)
    facts = sum(prog.full_count(h) for h in rels.values())
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches = 0
    with ClockSampler(local_rank) as clocks:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            starts[i].record(stream)
            prog.execute(batch)
            ends[i].record(stream)
            launches += prog.stats().kernel_launches
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms, facts_all = reduce_ranks(sum(step_ms), facts, f"cuda:{local_rank}")
    value = facts_all * args.steps / (total_ms / 1e3)
    st = prog.stats()
    # device time per phase of the wide iteration (per-launch events, one extra run)
    prog.set_launch_timing(True)
    prog.execute(batch)
    ph = prog.stats().phase_ms
    prog.set_launch_timing(False)
    names = ("join ranges + scan", "plan", "candidates (join expand / copy)", "winners (sort + dedup)",
             "newt (ids + sort)", "full + delta merge")
    phases = {n: round(v, 3) for n, v in zip(names, ph) if n != "plan"}
    # end to end through the C ABI: every relation from pinned host rows, then history + counts back
    pinned = {n: torch.from_numpy(r.view(np.int64)).pin_memory().numpy().view(np.uint64) for n, r in host_rows.items()}
    e2e_s = []
    for _ in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for n, r in pinned.items():
            prog.load_rows(rels[n], r)
        prog.execute(batch)
        hist = prog.history()
        got = sum(prog.full_count(h) for h in rels.values())
        e2e_s.append(time.perf_counter() - t0)
        assert got == facts
    h2d = int(sum(r.nbytes for r in host_rows.values()))
    d2h = 8 * (2 * len(rels) + sum(2 + 2 * len(x[1]) for x in hist))
    e2e_ms, e2e_units = reduce_ranks(1e3 * statistics.mean(e2e_s), facts, f"cuda:{local_rank}")
    e2e = {"value": e2e_units / (e2e_ms / 1e3), "unit": "facts/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": int(d2h)}
    peak, peak_kind = load_peaks()
    dom = max(phases, key=phases.get)
    if rank != 0:
        return None
    line = {
        "metric": "facts/s", "value": value, "unit": "facts/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "the reference's own input relations (tests/golden fixtures)",
        "config": {"workload": args.workload, "program": DESCRIBED[args.workload], "batch_size": batch,
                   "output_facts": facts, "iterations": int(st.iterations), "join_candidates": int(st.join_candidates),
                   "path": "wide tuples (rows of u64 columns, trie order)",
                   "l2": "flushed (256 MiB write) before every timed step",
                   "phase_ms_per_run": phases, "parallelism": f"{world} independent instance(s), one per GPU",
                   "metric_family": METRIC_FAMILY},
        "clocks": clocks.summary(), "e2e": e2e, "gpu_launches": int(launches),
        "roofline": {"kernel": dom, "bound": "latency", "achieved": None, "peak": peak, "unit": "GB/s",
                     "frac": None, "peak_kind": peak_kind, "traffic": None,
                     "note": f"{int(st.kernel_launches)} launches per run over {int(st.iterations)} iterations of "
                             f"small deltas: launch- and synchronisation-bound, not HBM-bound"},
        "step_ms": step_ms,
    }
    if world == 1 and not args.no_cpu_baseline:
        rf, rs = described_reference_run(args.workload)
        assert rf == facts
        line["cpu_baseline"] = {"value": rf / rs, "unit": "facts/s", "cores": 1, "kind": "reference",
                                "sample": f"the whole program on the reference library (fixpoint {rs:.1f} s)"}
    return line


BATCH_COUNT, BATCH_SEED = 8192, 1
BATCH_SERIAL_SAMPLE = 512
BATCH_CPU_SAMPLE = 12


def gen_processes():
    return max(1, min(32, (os.cpu_count() or 2) - 1))


def batched_instances(count, seed):
    """The batched workload: per-instance seeded ER graphs (datagen.batched_sizes)."""
    import parallel_ra_b200 as P
    return P.datagen.generate_many([("er", n, m, s) for n, m, s in P.datagen.batched_sizes(count, seed)],
                                   gen_processes())


def batched_cpu_baseline(insts, total_tuples):
    """Reference CPU throughput on a bounded random sample of the batch (instances whose
    closure is estimated below 5e6 tuples), converted to instances/s over the whole batch."""
    from parallel_ra_b200.batch import estimate_tuples
    rng = np.random.default_rng(7)
    pool = [i for i in rng.permutation(len(insts)) if estimate_tuples("tc", insts[i]) < 5e6][:BATCH_CPU_SAMPLE]
    tup = secs = 0.0
    kind = "port"
    for i in pool:
        t, sec, kind = reference_rows_run(insts[i])
        tup += t
        secs += sec
    tps = tup / secs
    return {"value": len(insts) / (total_tuples / tps), "unit": "instances/s", "cores": 1, "kind": kind,
            "tuples_per_s": tps,
            "sample": f"{len(pool)} random instances of the batch with estimated closure < 5e6 tuples "
                      f"({int(tup)} tuples, {secs:.1f} s fixpoint time); instances/s = batch size / "
                      f"(batch tuples / sample tuples/s)"}


def run_batched(args, rank, world, local_rank):
    """8,192 independent TC instances (n log-uniform in [64, 16384], mean out-degree
    uniform in [0.8, 2.0]) run as waves of rebased unions -- one CUDA-graph-driven
    program per wave -- against plain one-instance-per-run executions."""
    import torch
    import parallel_ra_b200 as P
    from parallel_ra_b200.batch import Runner, estimate_tuples, plan_waves, value_span

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    insts = batched_instances(BATCH_COUNT, BATCH_SEED + 1000 * rank)
    est = np.array([estimate_tuples("tc", r) for r in insts])
    order = np.argsort(-est, kind="stable")
    free, _ = torch.cuda.mem_get_info(local_rank)
    budget = args.wave_tuples or min(P.batch.WAVE_TUPLES, 0.5 * free / P.batch.BYTES_PER_TUPLE)
    spans = [value_span(insts[i]) for i in order]
    # waves within the tuple budget, the 30-bit join-key range and the dense evaluator's bit matrices
    waves = [[int(order[j]) for j in w] for w in plan_waves(est[order], budget, max_values=(1 << 30) - 1,
                                                             spans=spans,
                                                             max_dense_bytes=0.9 * P.batch.DENSE_MAX_BYTES)]
    stream = torch.cuda.Stream()
    runner = Runner("tc", local_rank)
    runner.prog.set_stream(stream.cuda_stream)
    # union rows of every wave resident in HBM before timing
    staged = []
    for w in waves:
        union, base = Runner.union_rows([insts[i] for i in w])
        staged.append((w, base, torch.from_numpy(union.view(np.int64)).to(dev), union.shape[0]))
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)

    def one_pass():
        res, launches, tuples, peak = {}, 0, 0, 0
        for w, base, t, nrows in staged:
            out = runner.run_wave_resident(base, t.data_ptr(), nrows)
            st = runner.prog.stats()
            launches += st.kernel_launches
            peak = max(peak, st.device_bytes_peak)
            for i, o in zip(w, out):
                res[i] = o
                tuples += o.counts["T"]
        return res, launches, tuples, peak

    for _ in range(args.warmup):
        one_pass()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    step_ms, launches = [], 0
    with ClockSampler(local_rank) as clocks:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            res, launches, tuples, peak = one_pass()
            b.record(stream)
            torch.cuda.synchronize()
            step_ms.append(a.elapsed_time(b))
    if world > 1:
        torch.distributed.barrier()
    # whole job: every rank's batch (its own instances) over the slowest rank's device time
    total_ms, done = reduce_ranks(sum(step_ms), BATCH_COUNT * args.steps, dev)
    value = done / (total_ms / 1e3)

    # dominant kernel on the largest wave, with per-launch events
    w, base, t, nrows = staged[0]
    runner.prog.set_launch_timing(True)
    runner.run_wave_resident(base, t.data_ptr(), nrows)
    s2 = runner.prog.stats()
    runner.prog.set_launch_timing(False)
    dense = {"search_ms": 0.0, "emit_ms": 0.0, "sccs": 0, "new_tuples": 0, "candidates": 0}
    accumulate_dense(dense, s2)
    peak_bw, peak_kind = load_peaks()
    achieved = (s2.dedup_bytes / s2.dedup_launches) / ((s2.dedup_ms / s2.dedup_launches) / 1e3) / 1e9 \
        if s2.dedup_launches else 0.0
    if dense["sccs"]:
        roofline = dense_roofline(dense, peak_bw, peak_kind)
        roofline.update({"wave": "largest wave", "instances_in_wave": len(w)})
    else:
        roofline = {"kernel": "join_fused_kernel", "bound": "hbm", "achieved": achieved, "peak": peak_bw,
                    "unit": "GB/s", "frac": achieved / peak_bw, "peak_kind": peak_kind,
                    "traffic": TRAFFIC_PER_ALGO_BYTE * s2.dedup_bytes / max(s2.dedup_launches, 1),
                    "traffic_note": "ncu DRAM read+write per algorithmic byte measured on tc-er20, times this "
                                    "wave's algorithmic bytes per launch",
                    "launches": int(s2.dedup_launches), "wave": "largest wave", "instances_in_wave": len(w)}
    # end to end from host arrays: rebasing, upload, waves, per-instance results
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h2d = d2h = 0
    res_e2e = {}
    for w in waves:
        out = runner.run_wave([insts[i] for i in w])
        for i, o in zip(w, out):
            res_e2e[i] = o
        h2d += sum(insts[i].nbytes for i in w)
        hist_rows = sum(it for _, it in runner._scc_blocks())
        d2h += 8 * len(w) * (hist_rows + 2 * len(runner.rels))   # per-instance counts + (count, digest)
    e2e_s = time.perf_counter() - t0
    e2e_ms, e2e_done = reduce_ranks(1e3 * e2e_s, BATCH_COUNT, dev)
    runner.close()          # release its buffers before the plain runs

    # serial: plain one-instance-per-run executions of a random sample, each checked against its wave result
    sample = np.random.default_rng(3).choice(BATCH_COUNT, BATCH_SERIAL_SAMPLE, replace=False)
    plain = Runner("tc", local_rank)
    plain.run_plain(insts[int(sample[0])])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mismatches = 0
    for i in sample:
        o = plain.run_plain(insts[int(i)])
        mismatches += int(o.key() != res[int(i)].key() or o.key() != res_e2e[int(i)].key())
    serial_s = time.perf_counter() - t0
    plain.close()
    if mismatches:
        raise RuntimeError(f"{mismatches} batched instances differ from their plain runs")
    serial_ips = BATCH_SERIAL_SAMPLE / serial_s

    if rank != 0:
        return None
    iters = [sum(len(d) for d in res[i].deltas) for i in range(BATCH_COUNT)]
    line = {
        "metric": "batched TC instances/s", "value": value, "unit": "instances/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(step_ms) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": "batched", "instances": BATCH_COUNT, "seed": BATCH_SEED,
                   "sizes": "n log-uniform in [64, 16384], mean out-degree uniform in [0.8, 2.0]",
                   "waves": len(waves), "wave_tuple_budget": budget, "tc_tuples": int(tuples),
                   "tuples_per_s": tuples * args.steps / (sum(step_ms) / 1e3),
                   "peak_device_bytes": int(peak), "max_instance_iterations": int(max(iters)),
                   "l2": "flushed (256 MiB write) before every timed step; waves are larger than L2",
                   "step": "every wave of the batch, union rows resident in HBM, per-instance results to host",
                   "metric_family": METRIC_FAMILY},
        "serial": {"value": serial_ips, "unit": "instances/s", "sample": int(BATCH_SERIAL_SAMPLE),
                   "mode": "plain one-instance-per-run executions (one reused program) from host rows, "
                           "random sample of the batch",
                   "batched_e2e_over_serial": (BATCH_COUNT / e2e_s) / serial_ips,
                   "bit_exact_mismatches": mismatches},
        "clocks": clocks.summary(),
        "e2e": {"value": e2e_done / (e2e_ms / 1e3), "unit": "instances/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches), "roofline": roofline, "step_ms": step_ms,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = batched_cpu_baseline(insts, tuples)
    return line


SERVED_COUNT, SERVED_SEED = 20000, 4
SERVED_RATES = (100.0, 1000.0, 10000.0)
SERVED_RATES_DEFAULT = SERVED_RATES
SERVED_POINT_SECONDS = 10.0
SERVED_CHECK_SAMPLE = 400


def run_served(args, rank, world, local_rank, rates=SERVED_RATES_DEFAULT):
    """Open-loop Poisson request streams (80% TC, 20% SG, 2% large TC) against the
    continuous-batching server, swept over arrival rates; latency percentiles and
    instances/s per rate, every checked result equal to a plain single-instance run."""
    import torch
    import parallel_ra_b200 as P
    from parallel_ra_b200.serve import Request, Server, poisson_arrivals, request_mix, run_stream

    torch.cuda.set_device(local_rank)
    reqs = request_mix(SERVED_COUNT, SERVED_SEED + 1000 * rank, processes=gen_processes())
    from parallel_ra_b200.batch import estimate_tuples
    for r in reqs:
        r.est_tuples = estimate_tuples(r.kind, r.rows)

    def clones(sub):
        return [Request(r.rid, r.kind, r.rows, est_tuples=r.est_tuples) for r in sub]

    server = Server(local_rank, slots=args.slots, budget_bytes=args.budget_gb * 1e9)
    for _ in range(args.warmup):               # warm-up streams: graphs, buffers, learnt estimates
        run_stream(server, clones(reqs[:500]), poisson_arrivals(500, max(rates), 99))
    points = []
    top = None
    with ClockSampler(local_rank) as clocks:
        for rate in rates:
            k = SERVED_COUNT if rate == max(rates) else min(SERVED_COUNT, int(rate * SERVED_POINT_SECONDS))
            stream = clones(reqs[:k])
            w0 = len(server.waves)
            if world > 1:
                torch.distributed.barrier()   # every rank's server starts its stream together
            st = run_stream(server, stream, poisson_arrivals(k, rate, 7))
            waves = server.waves[w0:]
            st["rate"] = rate
            st["waves"] = len(waves)
            st["mean_wave_size"] = float(np.mean([w.size for w in waves]))
            st["gpu_launches"] = int(sum(w.launches for w in waves))
            st["max_held_gb"] = max(w.held_bytes for w in waves) / 1e9
            points.append(st)
            if rate == max(rates):
                top = (stream, st)
    server.close()

    # every sampled result of the top-rate stream equals its plain single-instance run
    stream, st_top = top
    rng = np.random.default_rng(11)
    sample = rng.choice(len(stream), min(SERVED_CHECK_SAMPLE, len(stream)), replace=False)
    plain = {"tc": P.batch.Runner("tc", local_rank), "sg": P.batch.Runner("sg", local_rank)}
    mismatches = sum(int(stream[int(i)].result is None or stream[int(i)].result.key() != plain[
        stream[int(i)].kind].run_plain(stream[int(i)].rows).key()) for i in sample)
    for r in plain.values():
        r.close()
    if mismatches:
        raise RuntimeError(f"{mismatches} served results differ from their plain runs")

    # the same stream served one instance at a time (no batching, one worker)
    one = Server(local_rank, slots=1, budget_bytes=args.budget_gb * 1e9, max_wave_requests=1)
    k1 = 1500
    st_one = run_stream(one, clones(reqs[:k1]), poisson_arrivals(k1, max(rates), 7))
    one.close()
    # whole job: every rank's top-rate stream over the slowest rank's serving time
    top_ms, served = reduce_ranks(1e3 * st_top["seconds"], len(stream), f"cuda:{local_rank}")
    if rank != 0:
        return None
    h2d = int(sum(r.rows.nbytes for r in stream))
    line = {
        "metric": "served instances/s", "value": served / (top_ms / 1e3), "unit": "instances/s",
        "n_gpus": world, "steps": 1, "warmup": args.warmup, "ms_per_step": top_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": "served", "requests": SERVED_COUNT, "seed": SERVED_SEED,
                   "mix": "80% TC (ER, n log-uniform [64, 16384], degree U[0.8, 2.0]), 20% SG (random trees, "
                          "n log-uniform [64, 16384]), 2% of all requests large TC (ER n=2^18, degree 0.95)",
                   "slots": args.slots, "budget_gb": args.budget_gb, "rates": points,
                   "p50_ms": st_top["p50_ms"], "p95_ms": st_top["p95_ms"], "p99_ms": st_top["p99_ms"],
                   "timing": "host wall clock from each request's submission to its results on the host; "
                             "step = the whole top-rate stream",
                   "metric_family": METRIC_FAMILY},
        "one_at_a_time": {"value": st_one["instances_per_s"], "unit": "instances/s", "requests": k1,
                          "p50_ms": st_one["p50_ms"], "p99_ms": st_one["p99_ms"],
                          "mode": "same server, one worker, waves of one request (plain runs)"},
        "admission": {"oom_retries": int(server.oom_retries), "unserved": int(sum(r.error is not None for r in stream)),
                      "learnt_bytes_per_tuple": server.bpt, "learnt_size_correction": server.correction},
        "bit_exact": {"checked": int(len(sample)), "mismatches": mismatches,
                      "against": "plain single-instance runs of the same requests"},
        "clocks": clocks.summary(),
        "e2e": {"value": served / (top_ms / 1e3), "unit": "instances/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": int(8 * 4 * len(stream))},
        "gpu_launches": int(st_top["gpu_launches"]),
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tc-er22",
                    choices=sorted(WORKLOADS) + sorted(DESCRIBED) + ["batched", "served"])
    ap.add_argument("--slots", type=int, default=4, help="served: concurrent waves (worker threads)")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="served: device-memory admission budget")
    ap.add_argument("--wave-tuples", type=float, default=0.0,
                    help="batched: estimated derived tuples per wave (default: the autotuned size, "
                         "capped by half the free device memory)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="tc-er22: leave out the bounded batched and served sub-records of config")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        if args.impl == "ours":
            torch.cuda.set_device(local_rank % max(1, torch.cuda.device_count()))
            # the ranks exchange only host-side scalars and histories: NCCL by default, or
            # RA_BENCH_BACKEND=gloo (e.g. several ranks sharing one GPU in a smoke run)
            dist.init_process_group(os.environ.get("RA_BENCH_BACKEND", "nccl"), timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        line = run_reference_arm(args, rank, world)
    elif args.workload in ("batched", "served"):
        line = (run_batched if args.workload == "batched" else run_served)(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    elif args.workload in DESCRIBED:
        line = run_described_ours(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    else:
        line = run_ours(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if line is not None and rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
