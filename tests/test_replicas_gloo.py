"""Multi-rank path of bench.py on CPU (gloo, world_size 2): replicas only -- each rank times its own
batch, the reported time is the slowest rank's and the throughput counts every rank's gates."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import replica_throughput
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [100.0, 250.0][rank]  # rank 1 is the slow one
        slowest, value = replica_throughput(local_ms, 4096, world, dist, "cpu")
        out[rank] = (slowest, value)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_uses_the_slowest_rank_gloo():
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    for rank in (0, 1):
        slowest, value = out[rank]
        assert slowest == pytest.approx(250.0)
        assert value == pytest.approx(2 * 4096 / 0.25)


def test_replica_throughput_single_rank():
    from bench import replica_throughput
    slowest, value = replica_throughput(50.0, 1000, 1)
    assert slowest == 50.0 and value == pytest.approx(20000.0)
