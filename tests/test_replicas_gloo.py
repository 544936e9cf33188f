"""Replica path of bench.py on CPU: two gloo ranks, max over ranks, seeds, sharding."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from lbm_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    d = replicas.init("gloo", timeout_s=30)
    try:
        r, lr, w = replicas.env_rank()
        d.barrier()
        m = replicas.max_over_ranks(10.0 * (rank + 1))
        out.put((rank, r, w, m, replicas.replica_seed(7, rank), replicas.shard(10, world, rank)))
        d.barrier()
    finally:
        d.destroy_process_group()


def test_two_rank_gloo_replicas():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1]
    assert all(x[2] == world for x in res)
    assert all(x[3] == 20.0 for x in res)                  # max over ranks seen by every rank
    assert res[0][4] != res[1][4]                          # distinct replica seeds
    members = sorted(res[0][5] + res[1][5])
    assert members == list(range(10))                      # every member on exactly one rank


def test_single_process_helpers():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.shard(5, 1, 0) == [0, 1, 2, 3, 4]
    with pytest.raises(Exception):
        replicas.shard(5, 0, 0)
