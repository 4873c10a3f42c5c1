"""Golden vectors of the reference's generated analyses (wide tuples).

For each program below, from the reference tree (--ref, or oracle/Makefile's
default, which $RA_REFERENCE overrides):
  * parses tests/<program>.cpp -- generated code with one statement per
    relation, SCC, rule and dependency -- into a program description
    tests/golden/<program>/program.txt (format in oracle/programs.h);
  * copies the relation files it reads from data/<dir>/ into
    tests/golden/<program>/data/ (fixtures);
  * runs the description on the reference library through
    oracle/_ref/ref_driver and records, as tests/golden/<program>.json, the
    per-SCC history of (sum |delta|, sum |full|), every relation's full count,
    a SHA-256 of its rows in trie order (data columns + intern id) and of its
    data columns, and the rows of small relations verbatim;
  * where the program source compiles against the reference library, builds
    and runs it unchanged and records the relation sizes it prints.

The copy_filter lambdas are recognised from their text (comparisons of
columns 0 and 1).  Run from the repo root:
    python tests/golden/make_slog_golden.py [--ref <parallel-RA checkout>]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
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
PROGRAMS = ["cfa-4-4-64", "worstcase-110-terms-4-m"]
VERBATIM_MAX_ROWS = 512

LAMBDAS = {
    "return !(data[0] == data[1]);": "ne", "return data[0] != data[1];": "ne",
    "return data[0] == data[1];": "eq", "return !(data[0] != data[1]);": "eq",
}


def rows_digest(rows: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(rows, dtype="<u8").tobytes()).hexdigest()


def split_args(s: str) -> list[str]:
    """Top-level comma split (braces and parentheses nest)."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    out.append(cur.strip())
    return out


def parse_program(src: str):
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)          # block comments
    src = re.sub(r"^\s*//.*$", "", src, flags=re.M)          # whole-line comments
    rels, rel_index = [], {}
    for m in re.finditer(r'relation\*\s+(\w+)\s*=\s*new relation\((\d+),\s*(true|false),\s*(\d+),\s*(\d+),\s*'
                         r'"([^"]*)",\s*"([^"]*)",\s*(FULL|DELTA)\)', src):
        var, jcc, canon, arity, tag, name, path, ver = m.groups()
        rel_index[var] = len(rels)
        rels.append(dict(jcc=int(jcc), canon=canon == "true", arity=int(arity), tag=int(tag), name=name,
                         path=path, ver=ver))
    ram = {}
    for m in re.finditer(r'RAM\*\s+(\w+)\s*=\s*new RAM\((true|false),\s*(\d+)\)', src):
        ram[m.group(1)] = (m.group(2) == "true", int(m.group(3)))
    order = re.findall(r'lie->add_scc\((\w+)\)', src)          # LIE's SCC order
    scc_index = {v: i for i, v in enumerate(order)}
    lines = ["batch %s" % (re.search(r'set_batch_size\((\d+)\)', src) or [None, "1"])[1]]
    for r in rels:
        lines.append("rel %d %d %d %d %s %s %s" % (r["jcc"], r["canon"], r["arity"], r["tag"], r["ver"], r["name"],
                                                   os.path.basename(r["path"]) or "-"))
    for v in order:
        lines.append("scc %d %d" % (1 if ram[v][0] else 0, ram[v][1]))
    for m in re.finditer(r'(\w+)->add_relation\((\w+),\s*(true|false)\)', src):
        if m.group(1) in scc_index:
            lines.append("member %d %d %d" % (scc_index[m.group(1)], rel_index[m.group(2)], m.group(3) == "true"))
    for m in re.finditer(r'(\w+)->add_rule\(new (parallel_\w+)\((.*?)\)\);\s*$', src, re.M):
        s = scc_index[m.group(1)]
        kind, a = m.group(2), split_args(m.group(3))
        cols = ",".join(x.strip() for x in a[-1 if kind != "parallel_copy_filter" else -2].strip("{}").split(","))
        if kind == "parallel_join":
            lines.append("join %d %d %d %s %d %s %s" % (s, rel_index[a[0]], rel_index[a[1]], a[2], rel_index[a[3]],
                                                       a[4], cols))
        elif kind in ("parallel_copy", "parallel_acopy"):
            lines.append("copy %d %s %d %d %s - %s" % (s, "copy" if kind == "parallel_copy" else "acopy",
                                                      rel_index[a[0]], rel_index[a[1]], a[2], cols))
        elif kind == "parallel_copy_filter":
            body = re.search(r'\{\s*(return[^;]*;)\s*\}', a[-1]).group(1)
            lines.append("copy %d filter %d %d %s %s %s" % (s, rel_index[a[0]], rel_index[a[1]], a[2],
                                                           LAMBDAS[re.sub(r"\s+", " ", body)], cols))
        else:
            raise ValueError(kind)
    for a, b in re.findall(r'lie->add_scc_dependance\((\w+),\s*(\w+)\)', src):
        lines.append("dep %d %d" % (scc_index[a], scc_index[b]))
    return lines, rels


def run_reference(desc: str, data_dir: str, work: str):
    empty = os.path.join(work, "empty_rel")
    P.datagen.write_empty_relation(empty)
    out = os.path.join(work, "out")
    t0 = time.time()
    subprocess.run([DRIVER, "file", desc, empty, out, data_dir], check=True, stdout=subprocess.DEVNULL)
    wall = time.time() - t0
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
    fix = float(open(os.path.join(out, "time.txt")).read())
    return hist, rels, fix, wall


def printed_sizes(prog: str, ref: str, data_dir: str, work: str):
    """The size lines the unchanged program prints on the reference library
    (None when the source does not compile there)."""
    exe = os.path.join(work, prog)
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-DNDEBUG", "-w", "-I", os.path.join(ROOT, "oracle", "mpi_shim"),
                        "-I", os.path.join(ref, "src"), os.path.join(ref, "tests", prog + ".cpp"),
                        os.path.join(ROOT, "oracle", "_ref", "libparallel_RA_ref.a"), "-o", exe],
                       capture_output=True)
    if r.returncode:
        return None
    run = os.path.join(work, "run")
    os.makedirs(os.path.join(work, "data"), exist_ok=True)
    os.makedirs(run, exist_ok=True)
    src = open(os.path.join(ref, "tests", prog + ".cpp")).read()
    sub = re.search(r'"\.\./data/([^/"]+)/', src).group(1)
    os.symlink(os.path.abspath(data_dir), os.path.join(work, "data", sub))
    out = subprocess.run([exe], cwd=run, capture_output=True, text=True, check=True).stdout
    return [ln for ln in out.splitlines() if "total facts" in ln or ln.startswith("Total facts")]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=O.reference_root(),
                    help="parallel-RA checkout (default: oracle/Makefile's, $RA_REFERENCE)")
    ap.add_argument("programs", nargs="*", default=PROGRAMS)
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={args.ref}", "-j8"], check=True)
    for prog in args.programs:
        src = open(os.path.join(args.ref, "tests", prog + ".cpp")).read()
        lines, rels = parse_program(src)
        dst = os.path.join(HERE, prog)
        os.makedirs(os.path.join(dst, "data"), exist_ok=True)
        with open(os.path.join(dst, "program.txt"), "w") as f:
            f.write(f"# generated from the reference's tests/{prog}.cpp by make_slog_golden.py\n")
            f.write("\n".join(lines) + "\n")
        for r in rels:
            base = os.path.basename(r["path"])
            srcf = os.path.normpath(os.path.join(args.ref, "tests", r["path"]))
            for suffix in ("", ".size"):
                shutil.copyfile(srcf + suffix, os.path.join(dst, "data", base + suffix))
        with tempfile.TemporaryDirectory() as work:
            hist, rel_out, fix, wall = run_reference(os.path.join(dst, "program.txt"), os.path.join(dst, "data"), work)
            printed = printed_sizes(prog, args.ref, os.path.join(dst, "data"), work)
        case = {"program": prog, "history": hist, "relations": rel_out,
                "reference_fixpoint_seconds_1core": round(fix, 3), "printed_sizes": printed}
        with open(os.path.join(HERE, f"{prog}.json"), "w") as f:
            json.dump(case, f, separators=(",", ":"))
        print(prog, "relations", len(rel_out), "facts", sum(v["count"] for v in rel_out.values()),
              "iterations", sum(len(h[1]) for h in hist), "fixpoint %.1f s (wall %.1f s)" % (fix, wall))


if __name__ == "__main__":
    main()
