"""The benchmark's multi-GPU plumbing on CPU ranks (gloo, world size 2):
each rank steps its own replica, the device time of the run is the slowest
rank's (max over ranks, every rank taking part), and the whole-job rate
counts every rank's steps.  Replicas only: no data-path collective."""
from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        mine = 100.0 + 37.5 * rank  # this rank's device milliseconds
        slowest = bench.max_over_ranks(mine, torch.device("cpu"), ws)
        out[rank] = (slowest, bench.whole_job_rate(ws, 5, slowest))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_on_two_ranks():
    ws = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(ws, _free_port(), out), nprocs=ws, join=True, start_method="spawn")
        res = dict(out)
    for r in range(ws):
        slowest, rate = res[r]
        assert slowest == 137.5
        assert rate == pytest.approx(2 * 5 / 0.1375)


def test_single_rank_needs_no_process_group():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    assert bench.max_over_ranks(12.5, torch.device("cpu"), 1) == 12.5
    assert bench.whole_job_rate(1, 4, 500.0) == pytest.approx(8.0)
