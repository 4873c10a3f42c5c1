"""Transitive closure partitioned over ranks by the source column (partition.py).

* Two gloo ranks on the CPU, each running its partition on the CPU oracle:
  the history reduced across ranks and the union of the ranks' T equal a
  single-rank run of the reference's program.
* In one process, P = 1, 3 and 5 partitions combined the same way.
* On the GPU, the engine runs each partition in turn (no rank waits on
  another): the combined history and T equal one engine run of the program.
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
import parallel_ra_b200 as P
from parallel_ra_b200 import partition as PT

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def as_lists(hist):
    return [[sid, [list(x) for x in pairs]] for sid, pairs in hist]


def sorted_rows(rows):
    rows = np.ascontiguousarray(rows[:, :2])
    return rows[np.lexsort((rows[:, 1], rows[:, 0]))]


def single_oracle(rows):
    o = O.OracleProgram()
    rels = P.programs.build_tc(o, rows)
    o.execute(1)
    return o.history(), o.dump_full(rels["T"])


def graph():
    # near the critical degree: cycles, long paths and some duplicate-free hubs
    return P.datagen.with_row_ids(P.datagen.erdos_renyi(1500, 1600, 41))


def test_owner_spreads_values():
    v = np.arange(100000, dtype=np.uint64)
    for world in (2, 3, 8):
        counts = np.bincount(PT.owner(v, world), minlength=world)
        assert counts.min() > 0.9 * len(v) / world
    assert np.array_equal(PT.owner(v, 1), np.zeros(len(v), dtype=np.int64))


@pytest.mark.parametrize("world", [1, 3, 5])
def test_partitions_combine_to_the_single_rank_run(world):
    rows = graph()
    hist, T = single_oracle(rows)
    hists, parts = [], []
    for r in range(world):
        o = O.OracleProgram()
        rels = PT.build_tc_partitioned(o, rows, r, world)
        o.execute(1)
        hists.append(o.history())
        parts.append(o.dump_full(rels["T"]))
        # every tuple of rank r's T keeps a source rank r owns
        assert np.all(PT.owner(parts[-1][:, 1], world) == r)
    assert as_lists(PT.combine_histories(hists)) == as_lists(hist)
    assert np.array_equal(sorted_rows(np.concatenate(parts)), sorted_rows(T))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as Ol
    import parallel_ra_b200 as Pl
    from parallel_ra_b200 import partition as PTl
    rows = Pl.datagen.with_row_ids(Pl.datagen.erdos_renyi(1500, 1600, 41))
    o = Ol.OracleProgram()
    rels = PTl.build_tc_partitioned(o, rows, rank, world)
    o.execute(1)
    hist = PTl.global_history(o.history())
    parts = [None] * world
    dist.all_gather_object(parts, o.dump_full(rels["T"])[:, :2])
    if rank == 0:
        np.save(os.path.join(out_dir, "T.npy"), np.concatenate(parts))
        with open(os.path.join(out_dir, "hist.txt"), "w") as f:
            f.write(repr(as_lists(hist)))
    dist.destroy_process_group()


def test_two_gloo_ranks_equal_the_single_rank_run(tmp_path):
    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    hist, T = single_oracle(graph())
    assert open(tmp_path / "hist.txt").read() == repr(as_lists(hist))
    assert np.array_equal(sorted_rows(np.load(tmp_path / "T.npy")), sorted_rows(T))


def run_engine_partitions(rows, world, persist=False):
    hists, parts = [], []
    for r in range(world):
        p = P.Program(0)
        p.set_evaluators(reach=False, persistent=persist)
        rels = PT.build_tc_partitioned(p, rows, r, world)
        p.execute(1)
        hists.append(p.history())
        parts.append(p.dump_full(rels["T"]))
        p.close()
    return PT.combine_histories(hists), np.concatenate(parts)


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 4])
def test_engine_partitions_equal_one_engine_run(world):
    # above the dense evaluator's value range: the semi-naive hash-set path on every partition
    rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(200000, 199000, 42))
    p = P.Program(0)
    rels = P.programs.build_tc(p, rows)
    p.execute(1)
    hist, T = p.history(), p.dump_full(rels["T"])
    p.close()
    ph, pT = run_engine_partitions(rows, world, persist=world == 4)
    assert ph == hist
    assert np.array_equal(sorted_rows(pT), sorted_rows(T))
