"""Multi-process plumbing of bench.py's replica mode on the CPU (gloo,
world size 2): every rank gets the max over ranks of the step time and the
job value counts every rank's replica."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist

    import bench

    w, r, _ = bench.dist_setup()
    ms = bench.barrier_max(10.0 + 5.0 * r, w)  # rank 1 is the slow one
    bench.barrier(w)
    with open(os.path.join(out, f"r{r}"), "w") as f:
        f.write(f"{w} {ms}")
    dist.destroy_process_group()


def test_two_rank_max_over_ranks(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    port = _free_port()
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    got = sorted(open(tmp_path / f"r{r}").read().split() for r in range(2))
    assert got == [["2", "15.0"], ["2", "15.0"]]
