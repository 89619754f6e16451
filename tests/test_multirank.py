"""The multi-process plumbing of bench.py on CPU (gloo, world size 2): every
rank reports the slowest rank's time, and the whole-job rate counts the units
of all ranks over that time.  bench.py --gpus N runs N replicas, one process
per GPU, with this as its only collective."""
from __future__ import annotations

import json
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank: int, world: int, port: int, out_dir: str):
    import torch
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    times = [1.25, 3.5]  # this rank's own step time (rank 1 is the slow one)
    slowest = bench.max_over_ranks(times[rank], dist, torch.device("cpu"))
    rate = bench.whole_job_rate(10, world, slowest)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"slowest": slowest, "rate": rate}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    mp.spawn(worker, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True)
    got = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    for g in got:
        assert g["slowest"] == 3.5
        assert g["rate"] == pytest.approx(2 * 10 / 3.5)


def test_single_process_is_identity():
    import bench

    assert bench.max_over_ranks(2.5, None, None) == 2.5
    assert bench.whole_job_rate(7, 1, 0.5) == 14.0
