"""The multi-GPU path is independent replicas (no exchange step): ranks
only agree on the slowest rank's time.  Two gloo ranks on the CPU run the
same helpers bench.py uses under torchrun."""
from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, ws: int, port: int, q):
    import datetime

    import torch.distributed as dist

    from fuller_md_en_b200.replicas import job_throughput, max_over_ranks, replica_seed
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank                    # rank 1 is the slowest
        m = max_over_ranks(ms)
        q.put((rank, replica_seed(42, rank), m, job_throughput(30000, 100, m, ws)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replica_timing_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [42, 43]              # independent seeds
    assert all(r[2] == 15.0 for r in res)               # max over ranks on every rank
    assert all(abs(r[3] - 2 * 30000 * 100 / 0.015) < 1e-6 * r[3] for r in res)


def test_single_process_needs_no_group():
    from fuller_md_en_b200.replicas import job_throughput, max_over_ranks
    assert max_over_ranks(7.5) == 7.5
    assert job_throughput(10, 4, 2.0, 1) == 20000.0
