"""Checkpoint dumps and restart of the unchanged transitive_closure.cpp program
(`TC <edge> <output_dir> <every>` / `TC --restart <dump> <output_dir> <every>`):
the B200 build writes the same checkpoint directories as the reference built
here (oracle/_ref/TC), file for file and byte for byte (the reference's a2a_*
all-to-all metadata aside), and a restart from a dump finishes with the same
relations."""
import filecmp
import os
import subprocess

import numpy as np
import pytest

import parallel_ra_b200 as P
from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

OURS = os.path.join(ROOT, "parallel-ra_b200", "cxx", "bin", "TC")
REF = os.path.join(ROOT, "oracle", "_ref", "TC")


def layout(tmp):
    """cwd with ../data/g5955/path_2_1_2, the empty T relation TC loads by relative path."""
    P.datagen.write_empty_relation(os.path.join(tmp, "data", "g5955", "path_2_1_2"))
    run = os.path.join(tmp, "run")
    os.makedirs(run, exist_ok=True)
    return run


def run_tc(binary, args, cwd):
    env = dict(os.environ, RA_ID_ORDER="reference")
    r = subprocess.run([binary] + args, cwd=cwd, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def final_counts(out):
    return [l for l in out.splitlines() if "total facts" in l]


def dump_files(d):
    out = {}
    for cp in sorted(os.listdir(d)):
        for f in sorted(os.listdir(os.path.join(d, cp))):
            if not f.startswith("a2a"):
                out[(cp, f)] = os.path.join(d, cp, f)
    return out


def assert_same_dumps(a, b):
    fa, fb = dump_files(a), dump_files(b)
    assert sorted(fa) == sorted(fb)
    for k in fa:
        assert filecmp.cmp(fa[k], fb[k], shallow=False), k


def edge_file(tmp, case):
    if case == "g13236":
        return os.path.join(GOLDEN, "g13236_edge_2_1_2")
    path = os.path.join(tmp, "edge_er")
    P.datagen.write_relation(path, P.datagen.with_row_ids(P.datagen.erdos_renyi(300, 420, 4)))
    return path


@pytest.mark.parametrize("case,every", [("g13236", 1), ("g13236", 3), ("er300", 1), ("er300", 2)])
def test_checkpoint_dumps_match_reference(tmp_path, case, every):
    """The reference TC only runs with a dump every batch: with its all-to-all record on
    (TC enables it) it writes into checkpoint directories that exist every
    cp_iteration-th batch only, and crashes otherwise.  So it always dumps every batch
    here, and with every > 1 the B200 build's dumps are compared with the reference's
    dumps of the same batches."""
    if not os.path.exists(REF):
        pytest.skip("reference TC not built (oracle/Makefile)")
    tmp = str(tmp_path)
    run = layout(tmp)
    edge = edge_file(tmp, case)
    ref_out = run_tc(REF, [edge, os.path.join(tmp, "ref"), "1"], run)
    our_out = run_tc(OURS, [edge, os.path.join(tmp, "ours"), str(every)], run)
    assert final_counts(our_out) == final_counts(ref_out)
    ref = dump_files(os.path.join(tmp, "ref"))
    ours = dump_files(os.path.join(tmp, "ours"))
    ref = {k: v for k, v in ref.items() if int(k[0].rsplit("-", 1)[1]) % every == 0}
    assert sorted(ref) == sorted(ours)
    for k in ref:
        assert filecmp.cmp(ref[k], ours[k], shallow=False), k


@pytest.mark.parametrize("checkpoint", ["checkpoint-1-0", "checkpoint-1-4", "checkpoint-1-9"])
def test_restart_matches_reference(tmp_path, checkpoint):
    """(checkpoint-2-0, after the copy SCC, holds no T_full file -- T's full version is
    empty there -- and the reference cannot restart from it.)"""
    if not os.path.exists(REF):
        pytest.skip("reference TC not built (oracle/Makefile)")
    tmp = str(tmp_path)
    run = layout(tmp)
    edge = edge_file(tmp, "g13236")
    run_tc(REF, [edge, os.path.join(tmp, "first"), "1"], run)
    dump = os.path.join(tmp, "first", checkpoint)
    ref_out = run_tc(REF, ["--restart", dump, os.path.join(tmp, "ref"), "1"], run)
    our_out = run_tc(OURS, ["--restart", dump, os.path.join(tmp, "ours"), "1"], run)
    assert final_counts(our_out) == final_counts(ref_out)
    assert_same_dumps(os.path.join(tmp, "ref"), os.path.join(tmp, "ours"))


def test_restart_from_own_dump_finishes_the_closure(tmp_path):
    """Python API: dump every 2 batches (shared-file layout), restart from a mid-fixpoint
    dump in emission id order (dense evaluator allowed), same tuples as a straight run."""
    tmp = str(tmp_path)
    rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(400, 600, 9))
    p = P.Program(0)
    rels = P.programs.build_tc(p, rows)
    p.set_checkpoint(os.path.join(tmp, "cp"), 2)
    p.execute(1)
    want = p.dump_full(rels["T"])[:, :2]
    dump = os.path.join(tmp, "cp", "checkpoint-1-4")
    assert open(os.path.join(dump, "scc_metadata")).read().split() == ["2"]
    q = P.Program(0)
    T = q.relation(1, 2, 257, "T", P.engine.FULL)
    G = q.relation(1, 2, 256, "G", P.engine.FULL)
    q.load_file(T, os.path.join(dump, "T_full"))
    q.load_file(G, os.path.join(dump, "G_full"))
    join = q.scc(True, 1)
    q.add_relation(join, G, False)
    q.add_relation(join, T, True)
    q.join(join, T, T, P.engine.DELTA, G, P.engine.FULL, [3, 1])
    copy = q.scc(False, 2)
    q.add_relation(copy, G, False)
    q.add_relation(copy, T, True)
    q.copy(copy, T, G, P.engine.FULL, [1, 0])
    q.depend(copy, join)
    q.set_restart(dump)
    q.execute(1)
    assert np.array_equal(q.dump_full(T)[:, :2], want)
    assert [sid for sid, _ in q.history()] == [1]      # the copy SCC is not run again
