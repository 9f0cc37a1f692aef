"""The multi-GPU bench path is replicas only (each rank screens its own copy of the workload; no
exchange on the data path): its host plumbing -- barrier, max-over-ranks timing and the
whole-job aggregate -- runs here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        bench.barrier(world)
        local_ms = 10.0 + 5.0 * rank            # rank 1 is the slow one
        slowest = bench.max_over_ranks(local_ms, world)
        units = 1000                            # per-rank work: fixed as N grows (weak scaling)
        out[rank] = (slowest, units * world / (slowest / 1e3))
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_aggregate():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        port = free_port()
        procs = [ctx.Process(target=worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[0] == out[1] == (15.0, 2000 / 0.015)
