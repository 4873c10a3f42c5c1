"""Autotuner for the engine's runtime knobs (``ra_tuning``) and the wave size
of batched runs.

What it picks, by measurement on the GPU it runs on:

* ``seen_load_max`` -- hash load factor of the seen sets (slots per stored
  tuple = 1 / load): lower loads mean shorter probe runs, higher ones a smaller
  table (fewer TLB misses, more of it in L2, less memory per tuple);
* ``seen_grow`` -- how far ahead a rebuilt seen set is sized (rebuilds vs memory);
* ``join_blocks_per_sm`` / ``select_blocks_per_sm`` -- CTA shape of the fused
  join kernel and of the winner selection (the kernels take tiles from a
  device counter, so any grid covers the work);
* ``wave_tuples`` -- estimated derived tuples per wave of a batched run.

Each candidate setting runs the calibration workloads (one large TC instance,
and one wave of the batched workload's instance mix) a few times; the score is
the median device-synchronised wall time of ``execute``.  Settings within 3% of
the best are broken by peak device memory.  The choice and the whole table go
to ``tuning.json`` beside the library; ``engine.Program`` applies that file
when it exists (``RA_TUNING_FILE`` names another; ``RA_TUNING_FILE=none``
skips it), and ``batch`` takes its wave size and bytes-per-tuple from it.

Run on the target GPU from the repository root:
    python -m parallel_ra_b200.autotune [--quick] [--out PATH]
"""
from __future__ import annotations

import argparse
import itertools
import json
import statistics
import time

from . import datagen
from .batch import Runner, estimate_tuples
from .engine import TUNING_PATH, Program
from .programs import build_tc

GRID = {
    "seen_load_max": (0.25, 0.35, 0.45, 0.55, 0.7),
    "seen_grow": (1.5, 2.5, 4.0),
    "join_blocks_per_sm": (4, 8),
    "select_blocks_per_sm": (4, 8),
}
QUICK_GRID = {
    "seen_load_max": (0.5, 0.65),
    "seen_grow": (2.0,),
    "join_blocks_per_sm": (4,),
    "select_blocks_per_sm": (4,),
}
WAVE_SIZES = (1e8, 2e8, 4e8)


def _timed(fn, reps, after_warm=None):
    import torch
    fn()
    torch.cuda.synchronize()
    if after_warm:
        after_warm()
    out = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        out.append(time.perf_counter() - t0)
    return statistics.median(out)


def calibration_single(scale: int):
    n = 1 << scale
    return datagen.with_row_ids(datagen.erdos_renyi(n, round(0.95 * n), 2))


def calibration_wave(target_tuples: float, seed: int = 5):
    """Instances of the batched mix (datagen.batched_sizes) up to ~target derived tuples."""
    insts, tot = [], 0.0
    for n, m, s in datagen.batched_sizes(4096, seed):
        rows = datagen.with_row_ids(datagen.erdos_renyi(n, m, s))
        e = estimate_tuples("tc", rows)
        if tot + e > target_tuples and insts:
            continue
        insts.append(rows)
        tot += e
        if tot > 0.9 * target_tuples:
            break
    return insts


def tune(grid, scale=20, wave_target=1.5e8, reps=3, device=0, log=print):
    single = calibration_single(scale)
    wave = calibration_wave(wave_target)
    prog = Program(device)
    rels = build_tc(prog, single)
    runner = Runner("tc", device)
    union, base = Runner.union_rows(wave)
    rows = []
    keys = list(grid)
    for combo in itertools.product(*(grid[k] for k in keys)):
        kw = dict(zip(keys, combo))
        # every setting starts from released buffers: the warm-up run grows them under its policy
        peaks = {"single": 0, "wave": 0}

        def peak(name, pr):
            peaks[name] = max(peaks[name], pr.stats().device_bytes_peak)
        prog.release()
        prog.set_tuning(**kw)
        runner.prog.release()
        runner.prog.set_tuning(**kw)
        t_single = _timed(lambda: prog.execute(1), reps, lambda: peak("single", prog))
        peak("single", prog)
        tc = prog.full_count(rels["T"])

        def run_wave():
            runner.declare(base)
            runner.prog.load_rows(runner.rels["G"], union)
            runner.prog.execute()
        t_wave = _timed(run_wave, reps, lambda: peak("wave", runner.prog))
        peak("wave", runner.prog)
        wave_tuples = runner.prog.full_count(runner.rels["T"])
        row = dict(kw, single_ms=1e3 * t_single, single_bytes_per_tuple=peaks["single"] / max(tc, 1),
                   wave_ms=1e3 * t_wave, wave_bytes_per_tuple=peaks["wave"] / max(wave_tuples, 1))
        rows.append(row)
        log(json.dumps(row))
    # score: sum of the two workloads' times relative to their best
    b1 = min(r["single_ms"] for r in rows)
    b2 = min(r["wave_ms"] for r in rows)
    for r in rows:
        r["score"] = r["single_ms"] / b1 + r["wave_ms"] / b2
    best = min(r["score"] for r in rows)
    near = [r for r in rows if r["score"] <= best * 1.03]
    pick = min(near, key=lambda r: r["single_bytes_per_tuple"] + r["wave_bytes_per_tuple"])
    chosen = {k: pick[k] for k in keys}
    prog.close()

    # wave size with the chosen knobs: throughput of the batched mix per budget
    runner.prog.set_tuning(**chosen)
    mix = calibration_wave(max(WAVE_SIZES) * 2, seed=9)
    est = [estimate_tuples("tc", r) for r in mix]
    wave_rows = []
    for budget in WAVE_SIZES:
        waves, cur, tot = [], [], 0.0
        for r, e in zip(mix, est):
            if cur and tot + e > budget:
                waves.append(cur)
                cur, tot = [], 0.0
            cur.append(r)
            tot += e
        if cur:
            waves.append(cur)

        held = [0]

        def run_all():
            for w in waves:
                runner.run_wave(w)
                held[0] = max(held[0], runner.prog.stats().device_bytes_peak)
        runner.prog.release()
        t = _timed(run_all, 1)
        wave_rows.append({"wave_tuples": budget, "seconds": t, "waves": len(waves), "peak_bytes": held[0]})
        log(json.dumps(wave_rows[-1]))
    best_w = min(wave_rows, key=lambda r: r["seconds"])
    runner.close()
    bpt = max(max(r["wave_bytes_per_tuple"] for r in rows if all(r[k] == chosen[k] for k in keys)),
              max(r["single_bytes_per_tuple"] for r in rows if all(r[k] == chosen[k] for k in keys)))
    return {"tuning": chosen, "wave_tuples": best_w["wave_tuples"], "bytes_per_tuple": bpt,
            "table": rows, "wave_table": wave_rows,
            "calibration": {"single": f"TC on ER n=2^{scale}, mean out-degree 0.95, seed 2",
                            "wave": f"{len(wave)} instances of the batched mix (~{wave_target:.3g} tuples)",
                            "reps": reps}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true", help="a two-point grid (smoke test of the tuner)")
    ap.add_argument("--out", default=TUNING_PATH)
    ap.add_argument("--scale", type=int, default=20)
    args = ap.parse_args()
    import torch
    res = tune(QUICK_GRID if args.quick else GRID, scale=args.scale)
    res["device"] = torch.cuda.get_device_name(0)
    res["written"] = time.strftime("%Y-%m-%d %H:%M:%S")
    with open(args.out, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps({k: res[k] for k in ("tuning", "wave_tuples", "bytes_per_tuple", "device")}))


if __name__ == "__main__":
    main()
