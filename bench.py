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
unchanged parallel-RA sources on a single-rank MPI stand-in) on a bounded
sample of the same graph family; see DESIGN.md.

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
    # name: (nodes, edges, seed)
    "tc-er22": (1 << 22, 3984589, 2),
    "tc-er20": (1 << 20, 996147, 2),        # same family at 1/4 scale (profiling case)
    "tc-er2000": (2000, 3000, 1),
}
# bounded CPU sample of the same graph family (mean out-degree 0.95)
CPU_SAMPLE = (1 << 17, round(0.95 * (1 << 17)), 2)
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (read + write) per algorithmic byte of join_fused_kernel, from the
# ncu capture in profiles/join_fused_kernel_tc-er20.md (1.79 / 1.81 / 1.83 over
# three launches of the same graph family at 1/4 scale); bench's `traffic` is
# this ratio times the algorithmic bytes of an average tc-er22 launch.
TRAFFIC_PER_ALGO_BYTE = 1.81


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


def reference_sample_run(n, m, seed):
    """Run the reference (oracle/_ref/ref_driver) once; returns (tc_tuples, seconds, kind)."""
    import parallel_ra_b200 as P
    rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(n, m, seed))
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if os.path.exists(drv):
        with tempfile.TemporaryDirectory() as tmp:
            edge, empty, out = (os.path.join(tmp, x) for x in ("edge", "empty", "out"))
            P.datagen.write_relation(edge, rows)
            P.datagen.write_empty_relation(empty)
            subprocess.run([drv, "tc", edge, empty, out], check=True, stdout=subprocess.DEVNULL)
            secs = float(open(os.path.join(out, "time.txt")).read())
            tc = next(int(l.split()[2]) for l in open(os.path.join(out, "sizes.txt")) if l.split()[0] == "T")
        return tc, secs, "reference"
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    p = O.OracleProgram()
    rels = P.programs.build_tc(p, rows)
    p.execute(1)
    return p.full_count(rels["T"]), p.fixpoint_seconds(), "port"


def cpu_sample_desc():
    n, m, s = CPU_SAMPLE
    return f"TC on ER n={n} m={m} seed={s} (same family as the workload, mean out-degree 0.95), fixpoint time only"


def run_reference_arm(args, rank, world):
    if rank != 0:
        return None
    n, m, s = CPU_SAMPLE
    vals = []
    for i in range(args.warmup + args.steps):
        tc, secs, kind = reference_sample_run(n, m, s)
        if i >= args.warmup:
            vals.append((tc, secs))
    tot_tc = sum(v[0] for v in vals)
    tot_s = sum(v[1] for v in vals)
    value = tot_tc / tot_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / len(vals), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": args.workload, "sample": cpu_sample_desc(), "metric_family": METRIC_FAMILY},
        "cpu_baseline": {"value": value, "unit": "tuples/s", "cores": 1, "kind": kind, "sample": cpu_sample_desc()},
        "e2e": {"value": value, "unit": "tuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def run_ours(args, rank, world, local_rank):
    import torch
    import parallel_ra_b200 as P

    torch.cuda.set_device(local_rank)
    n, m, seed = WORKLOADS[args.workload]
    seed = seed + 1000 * rank          # each rank: its own independent instance
    rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(n, m, seed))
    stream = torch.cuda.Stream()
    prog = P.Program(local_rank)
    prog.set_stream(stream.cuda_stream)
    rels = P.programs.build_tc(prog, rows)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=f"cuda:{local_rank}")

    for _ in range(args.warmup):
        prog.execute(1)
    tc = prog.full_count(rels["T"])
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
    total_ms = sum(step_ms)
    tc_all = tc
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{local_rank}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
        c = torch.tensor([tc], dtype=torch.float64, device=f"cuda:{local_rank}")
        torch.distributed.all_reduce(c, op=torch.distributed.ReduceOp.SUM)
        tc_all = int(c.item())
    value = tc_all * args.steps / (total_ms / 1e3)
    st = prog.stats()

    # dominant kernel (fused join count, scan, expansion + first-occurrence claim): per-launch
    # CUDA events on the engine's stream, in an instrumented pass over the same
    # program (the timed steps run as one CUDA graph, whose nodes events cannot split)
    prog.set_launch_timing(True)
    dedup_ms = dedup_bytes = dedup_launches = 0
    phase = [0.0] * 6
    for _ in range(max(1, min(args.steps, 3))):
        prog.execute(1)
        s2 = prog.stats()
        dedup_ms += s2.dedup_ms
        dedup_bytes += s2.dedup_bytes
        dedup_launches += s2.dedup_launches
        phase = [a + b for a, b in zip(phase, s2.phase_ms)]
    prog.set_launch_timing(False)

    # the same program with intern ids numbered exactly as the single-rank reference
    prog.set_id_order(P.engine.IDS_REFERENCE)
    ref_ms = []
    for _ in range(3):
        prog.execute(1)
        ref_ms.append(prog.stats().fixpoint_ms)
    prog.set_id_order(P.engine.IDS_EMISSION)

    # end to end through the C ABI from pinned host rows
    pinned = torch.from_numpy(rows.view(np.int64)).pin_memory()
    pinned_np = pinned.numpy().view(np.uint64)
    e2e_s = []
    d2h = 0
    for i in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        prog.load_rows(rels["G"], pinned_np)
        prog.load_rows(rels["T"], np.empty((0, 3), dtype=np.uint64))
        prog.execute(1)
        h = prog.history()
        f, _ = prog.counts(rels["T"])
        g, _ = prog.counts(rels["G"])
        e2e_s.append(time.perf_counter() - t0)
        d2h = 8 * (2 + sum(2 + 2 * len(x[1]) for x in h))
        assert f == tc
    e2e = {"value": tc / statistics.mean(e2e_s), "unit": "tuples/s", "h2d_bytes_per_step": int(rows.nbytes),
           "d2h_bytes_per_step": int(d2h)}

    peak, peak_kind = load_peaks()
    achieved = (dedup_bytes / dedup_launches) / ((dedup_ms / dedup_launches) / 1e3) / 1e9 if dedup_launches else 0.0
    roofline = {"kernel": "join_fused_kernel", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": TRAFFIC_PER_ALGO_BYTE * dedup_bytes / max(dedup_launches, 1),
                "traffic_note": "ncu DRAM read+write per launch, measured on tc-er20 and scaled by units processed",
                "launches": int(dedup_launches), "avg_launch_us": 1e3 * dedup_ms / max(dedup_launches, 1),
                "bytes_per_launch": dedup_bytes / max(dedup_launches, 1),
                "bytes_model": "48 B per candidate (8 B inner key read, 8 B candidate write, 16 B seen-slot read "
                               "+ 16 B write) + 24 B per outer delta row (key, row offset, CSR start)"}
    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": args.workload, "nodes": n, "edges": m, "seed": WORKLOADS[args.workload][2],
                   "tc_tuples": tc, "iterations": int(st.iterations), "join_candidates": int(st.join_candidates),
                   "value_bits": int(st.value_bits), "l2": "flushed (256 MiB write) before every timed step",
                   "id_order": "emission (default)",
                   "value_reference_ids": tc / (statistics.median(ref_ms) / 1e3),
                   "phase_ms_per_step": {k: v / max(1, min(args.steps, 3)) for k, v in
                                         zip(P.engine.Stats.PHASES, phase)},
                   "parallelism": f"{world} independent instance(s), one per GPU", "metric_family": METRIC_FAMILY},
        "clocks": clocks.summary(), "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline,
        "step_ms": step_ms,
    }
    if world == 1 and not args.no_cpu_baseline:
        ctc, csecs, kind = reference_sample_run(*CPU_SAMPLE)
        line["cpu_baseline"] = {"value": ctc / csecs, "unit": "tuples/s", "cores": 1, "kind": kind,
                                "sample": cpu_sample_desc()}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tc-er22", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        line = run_reference_arm(args, rank, world)
    else:
        line = run_ours(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if line is not None and rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
