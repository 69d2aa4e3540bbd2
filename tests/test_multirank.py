"""The multi-rank bookkeeping of bench.py, on CPU with the gloo backend.

Each rank scans its own shard (weak scaling, no data exchange); the timed
figure is the slowest rank's, and the job throughput counts every rank's
codes.  Two processes, world size 2, rendezvous on 127.0.0.1.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank          # rank 1 is the slow one
        ms = bench.max_over_ranks(local_ms, dist)
        value = bench.job_throughput(1000, 64, world, ms)
        out.put((rank, ms, value, bench.shard_seed(2, rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_and_throughput():
    import torch.multiprocessing as mp
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
    assert [r[1] for r in res] == [15.0, 15.0]             # max over ranks on both
    want = 2 * 64 * 1000 / (15.0e-3) / 1e9
    assert all(abs(r[2] - want) < 1e-12 for r in res)
    assert res[0][3] != res[1][3]                          # distinct shards


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.job_throughput(10_000_000, 64, 1, 100.0) == pytest.approx(6.4)
