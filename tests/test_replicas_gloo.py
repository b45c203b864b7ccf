"""The multi-GPU form is replicas (each rank renders its own frames, no data exchange). This
checks the benchmark's cross-rank logic with two gloo ranks on the CPU: the timing reduction
takes the slowest rank and the whole-job throughput counts every rank's frames."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    secs = [2.0, 3.5][rank]
    slowest = bench.max_over_ranks(secs, dist, "cpu")
    out[rank] = (slowest, bench.replica_throughput(2592000, 10, slowest, world))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replica_reduction():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    assert out[0][0] == out[1][0] == pytest.approx(3.5)
    assert out[0][1] == pytest.approx(2 * 2592000 * 10 / 3.5 / 1e9)
