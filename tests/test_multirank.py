"""Multi-GPU runs are replicas (gates are independent, no collective on the data path); the only
cross-rank step is the max-over-ranks step time. Exercised here with two gloo ranks on CPU."""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms, value = bench.aggregate(10.0 * (rank + 1), 16384, world)
    rc = bench.run_reference(type("A", (), {"gpus": world, "steps": 1, "warmup": 1})(), rank, world) \
        if rank == 1 else None
    q.put((rank, ms, value, rc))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value, rc in res:
        assert ms == pytest.approx(20.0)               # the slowest rank's step
        assert value == pytest.approx(2 * 16384 / 0.020)  # all ranks' gates over that step
    assert res[1][3] == 0  # the reference arm's non-zero ranks exit without work
