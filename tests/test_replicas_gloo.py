"""Multi-GPU form = independent replicas: the only cross-rank step is the
max-over-ranks timing reduction of bench.py.  Exercised with 2 gloo ranks on
the CPU (no GPU)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench

    got = bench.max_over_ranks(1.5 + rank, world, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got))


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 2.5, 1: 2.5}


def test_single_rank_identity():
    import bench

    assert bench.max_over_ranks(3.25, 1) == 3.25
