"""Multi-GPU runs of bench.py are independent replicas (a snapshot repair does
not shard): the job time is the maximum over ranks and the throughput counts
all ranks. Checked here with two gloo ranks on the CPU."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = [10.0, 14.0][rank]
    e2e = [11.0, 12.5][rank]
    res = bench.replica_totals(ms, e2e, 100_000, 20, 20, world, "cpu")
    out[rank] = res
    dist.destroy_process_group()


def test_replica_totals_max_over_ranks():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()  # no fork of this multi-threaded process
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        ms, e2e, value, e2e_value = out[r]
        assert ms == 14.0 and e2e == 12.5
        assert abs(value - 100_000 * 20 * 2 / 0.014) < 1e-3
        assert abs(e2e_value - 100_000 * 20 * 2 / 0.0125) < 1e-3
