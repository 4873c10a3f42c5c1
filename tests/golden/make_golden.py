"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs oracle/_ref/ref_driver (the unchanged parallel-RA sources built by
oracle/Makefile against a single-rank MPI stand-in) on
  * the reference's own fixtures data/g5955/edge_2_1_2 and
    data/g13236/edge_2_1_2 (copied here as fixtures), and
  * seeded synthetic graphs (TC on Erdos-Renyi graphs, SG on random trees),
and records, per case, the per-SCC history of (sum |delta|, sum |full|)
pairs, every relation's full count, a SHA-256 of each relation's sorted rows
(data columns + intern id) and one of its data columns alone.  Small
relations are also stored verbatim.

The LARGE cases are the benchmark's own inputs (transitive closure of the
2^22-node Erdos-Renyi graph, same generation on the 2^15-node random tree);
each takes minutes and gigabytes on one core, so they run only when named
with --only.  Their records also carry the reference's fixpoint seconds and
the driver's peak resident memory.

Needs the reference tree: --ref, or oracle/Makefile's default (which the
RA_REFERENCE environment variable overrides); run from the repo root:
    python tests/golden/make_golden.py [--ref <parallel-RA checkout>] [--only NAME ...]
On a machine without the tree but with oracle/_ref/ref_driver already built
there (a larger host, for a case whose reference run needs more memory), the
generated-input cases run with
    python tests/golden/make_golden.py --prebuilt --only NAME [--out DIR]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import resource
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import parallel_ra_b200 as P  # noqa: E402
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")

# (name, program, source) -- source is a reference fixture path or a generator spec
CASES = [
    ("g5955_tc", "tc", ("fixture", "g5955")),
    ("g13236_tc", "tc", ("fixture", "g13236")),
    ("er200_tc", "tc", ("er", 200, 300, 7)),
    ("er2000_tc", "tc", ("er", 2000, 3000, 1)),
    ("er20000_tc", "tc", ("er", 20000, 19000, 3)),
    ("tree256_sg", "sg", ("tree", 256, 11)),
    ("tree1024_sg", "sg", ("tree", 1024, 5)),
]
# the benchmark inputs: tc-er22 and sg-tree15 of bench.py
LARGE_CASES = [
    ("er4194304_tc", "tc", ("er", 1 << 22, 3984589, 2)),
    ("tree32768_sg", "sg", ("tree", 1 << 15, 3)),
]
VERBATIM_MAX_ROWS = 4096


def rows_digest(rows: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(rows, dtype="<u8").tobytes()).hexdigest()


def input_rows(src, ref_root):
    kind = src[0]
    if kind == "fixture":
        return P.datagen.read_relation(os.path.join(ref_root, "data", src[1], "edge_2_1_2"))
    if kind == "er":
        return P.datagen.with_row_ids(P.datagen.erdos_renyi(src[1], src[2], src[3]))
    if kind == "tree":
        return P.datagen.with_row_ids(P.datagen.random_tree(src[1], src[2]))
    raise ValueError(kind)


def run_reference(prog, edge_path, work):
    empty = os.path.join(work, "empty_rel")
    P.datagen.write_empty_relation(empty)
    out = os.path.join(work, "out")
    t0 = time.time()
    subprocess.run([DRIVER, prog, edge_path, empty, out], check=True, stdout=subprocess.DEVNULL)
    wall = time.time() - t0
    fixpoint = float(open(os.path.join(out, "time.txt")).read())
    hist = []
    for line in open(os.path.join(out, "history.txt")):
        a = line.split()
        if a[0] == "scc":
            hist.append([int(a[1]), []])
        else:
            hist[-1][1].append([int(a[0]), int(a[1])])
    rels = {}
    for line in open(os.path.join(out, "sizes.txt")):
        name, arity, count = line.split()
        arity, count = int(arity), int(count)
        rows = np.fromfile(os.path.join(out, name + ".bin"), dtype="<u8").reshape(-1, arity + 1)
        assert rows.shape[0] == count, (name, rows.shape, count)
        rels[name] = {"arity": arity, "count": count, "sha256": rows_digest(rows),
                      "data_sha256": rows_digest(rows[:, :arity])}
        if count <= VERBATIM_MAX_ROWS:
            rels[name]["rows"] = rows.tolist()
    return hist, rels, fixpoint, wall


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=O.reference_root(),
                    help="parallel-RA checkout (default: oracle/Makefile's, $RA_REFERENCE)")
    ap.add_argument("--only", nargs="*", help="run only these cases (LARGE cases run only when named)")
    ap.add_argument("--prebuilt", action="store_true",
                    help="use the ref_driver already built in oracle/_ref (a machine without the reference "
                         "tree); generated-input cases only")
    ap.add_argument("--out", default=HERE, help="directory for the case files (default: beside this script)")
    args = ap.parse_args()
    if args.prebuilt:
        if not os.path.exists(DRIVER):
            ap.error("--prebuilt: oracle/_ref/ref_driver is not built")
        if not args.only or any(src[0] == "fixture" for n, _, src in CASES + LARGE_CASES if n in args.only):
            ap.error("--prebuilt: name generated-input cases with --only")
    else:
        if not args.ref or not os.path.isdir(os.path.join(args.ref, "src")):
            ap.error("give the reference tree with --ref or RA_REFERENCE")
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={args.ref}", "-j8"],
                       check=True)
        for name in ("g5955", "g13236"):
            dst = os.path.join(HERE, f"{name}_edge_2_1_2")
            shutil.copyfile(os.path.join(args.ref, "data", name, "edge_2_1_2"), dst)
            shutil.copyfile(os.path.join(args.ref, "data", name, "edge_2_1_2.size"), dst + ".size")
    mpath = os.path.join(args.out, "manifest.json")
    manifest = json.load(open(mpath)) if os.path.exists(mpath) else {}
    cases = CASES + LARGE_CASES
    if args.only:
        cases = [c for c in cases if c[0] in args.only]
    else:
        cases = CASES
    for name, prog, src in cases:
        with tempfile.TemporaryDirectory() as work:
            rows = input_rows(src, args.ref)
            edge = os.path.join(work, "edge")
            P.datagen.write_relation(edge, rows)
            hist, rels, fixpoint, wall = run_reference(prog, edge, work)
        case = {"program": prog, "source": list(src), "input_rows": int(rows.shape[0]),
                "input_sha256": rows_digest(rows), "history": hist, "relations": rels}
        if (name, prog, src) in LARGE_CASES:
            case["reference_fixpoint_seconds_1core"] = round(fixpoint, 3)
            case["reference_wall_seconds_1core"] = round(wall, 3)
            case["reference_peak_rss_mb"] = round(resource.getrusage(resource.RUSAGE_CHILDREN).ru_maxrss / 1024)
        with open(os.path.join(args.out, f"{name}.json"), "w") as f:
            json.dump(case, f, separators=(",", ":"))
        manifest[name] = {k: case[k] for k in ("program", "source", "input_rows")}
        print(name, {r: v["count"] for r, v in rels.items()}, "iterations", [len(h[1]) for h in hist],
              "fixpoint %.1f s, wall %.1f s" % (fixpoint, wall), flush=True)
    with open(mpath, "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
