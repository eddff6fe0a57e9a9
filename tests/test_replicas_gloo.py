"""bench.py --gpus N runs N independent replicas (the path does not shard): the
aggregation takes the slowest rank's time and sums the ranks' cell-updates.
Checked with two gloo ranks on CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms, cells = bench.aggregate(10.0 + rank, 1000 * (rank + 1), world, device="cpu")
    q.put((rank, ms, cells))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, cells in res:
        assert ms == 11.0          # max over ranks
        assert cells == 3000.0     # sum over ranks


def test_single_rank_passthrough():
    import bench
    assert bench.aggregate(5.0, 7, 1) == (5.0, 7)
