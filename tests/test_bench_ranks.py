"""bench.py's whole-job figures of N independent replicas (one process per GPU;
here world size 2 over gloo on the CPU): every rank learns the slowest rank's
device time and the units all ranks processed, so `value` is the whole job's."""
import datetime
import os
import socket
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    ms, units = bench.reduce_ranks(10.0 * (rank + 1), 100 * (rank + 1), "cpu")
    with open(os.path.join(out_dir, f"rank{rank}"), "w") as f:
        f.write(f"{ms} {units}")
    dist.destroy_process_group()


def test_reduce_ranks_over_two_gloo_ranks(tmp_path):
    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        ms, units = open(tmp_path / f"rank{r}").read().split()
        assert float(ms) == 20.0 and int(units) == 300


def test_reduce_ranks_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_ranks(12.5, 7, "cpu") == (12.5, 7)
