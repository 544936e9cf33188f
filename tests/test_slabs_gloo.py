"""j-slab decomposition host logic on CPU: tile geometry, the neighbour ring of
m_mpi_decomp_init.F90:128-134, and the halo exchange over gloo ranks (2 ranks
in a ring, where each rank is both neighbours of the other, and 3 ranks with
and without periodic j)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from lbm_b200 import slabs


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, periodic, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method="env://")
    try:
        south, north = slabs.neighbours(rank, world, periodic)
        n = 12
        send_s = torch.full((n,), 100 * rank + 1, dtype=torch.uint8)      # plane j = 1, goes south
        send_n = torch.full((n,), 100 * rank + 2, dtype=torch.uint8)      # plane j = ny, goes north
        recv_s = torch.zeros(n, dtype=torch.uint8)
        recv_n = torch.zeros(n, dtype=torch.uint8)
        slabs.exchange(send_s, send_n, recv_s, recv_n, south, north)
        dist.barrier()
        out.put((rank, int(recv_s[0]), int(recv_n[0]), bool(torch.all(recv_s == recv_s[0])),
                 bool(torch.all(recv_n == recv_n[0]))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, True), (3, True), (3, False)])
def test_halo_exchange_over_gloo(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, periodic, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rs, rn, us, un in res:
        assert us and un
        south, north = slabs.neighbours(rank, world, periodic)
        # from the south: the south neighbour's plane j = ny; from the north: its plane j = 1
        assert rs == (100 * south + 2 if south is not None else 0) % 256
        assert rn == (100 * north + 1 if north is not None else 0) % 256


def test_tile_geometry():
    assert slabs.tile_rows(12, 3, 0) == (1, 4)
    assert slabs.tile_rows(12, 3, 2) == (9, 4)
    with pytest.raises(ValueError):
        slabs.tile_rows(10, 3, 0)                 # the reference stops: nyg /= ntiles*ny
    with pytest.raises(ValueError):
        slabs.tile_rows(12, 3, 3)
    assert slabs.neighbours(0, 4, True) == (3, 1)
    assert slabs.neighbours(3, 4, True) == (2, 0)
    assert slabs.neighbours(0, 4, False) == (None, 1)
    assert slabs.neighbours(3, 4, False) == (2, None)
    assert slabs.neighbours(0, 1, False) == (None, None)
    # a global array (nz+2, nyg+2, nx+2): tile r gets global rows j0-1 .. j0+ny, ghosts included
    a = np.arange(4 * 14 * 3).reshape(4, 14, 3)
    t1 = slabs.tile_slice(a, 1, 3)
    assert t1.shape == (4, 6, 3)
    assert np.array_equal(t1, a[:, 4:10])
    assert np.array_equal(slabs.tile_slice(a, 0, 3)[:, 0], a[:, 0])       # global ghost row 0
    assert np.array_equal(slabs.tile_slice(a, 2, 3)[:, -1], a[:, 13])     # global ghost row nyg+1
