"""Multi-rank plumbing on CPU: two gloo ranks (127.0.0.1)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gputrianglecounting_b200 import dist as gdist


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, size, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        assert gdist.world() == (rank, size)
        got = gdist.max_over_ranks(10.0 + rank * 5.0)
        own = list(gdist.shard(4096, rank, size))
        out.put((rank, got, own[0], own[-1], len(own)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_shards_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [15.0, 15.0]
    assert res[0][2:] == (0, 2047, 2048) and res[1][2:] == (2048, 4095, 2048)


def test_single_process_identity_and_uneven_shards():
    assert gdist.world() == (0, 1)
    assert gdist.max_over_ranks(3.5) == 3.5
    parts = [gdist.shard(10, r, 3) for r in range(3)]
    assert [len(p) for p in parts] == [4, 3, 3]
    assert sorted(i for p in parts for i in p) == list(range(10))
