"""j slabs over two gloo ranks with real halo planes (host only).

Each rank holds one j-tile of a small domain as reference-layout host arrays and
steps it with the oracle's routines in main.F90's order (postcoll, solids,
boundarycond per tile, then the halo exchange of m_mpi_halo_exchange_j.F90,
then drift and macrovars).  The planes j = 1 and j = ny travel in the byte
layout of lbm_halo_pack_j (lbm_b200.slabs.plane_from_ref, the host mirror of
the device plane; tests/test_gpu_slabs.py checks the mirror against the device
pack) through lbm_b200.slabs.exchange, and are unpacked into the ghost planes.

Checked: every received plane equals the row the neighbour packed (the south
neighbour's j = ny arrives as j = 0, the north neighbour's j = 1 as j = ny+1),
and after the steps each rank's tile equals, bit for bit, the same two tiles
stepped in one process with the planes copied directly."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from lbm_b200 import slabs
from lbm_b200 import workloads as W

WL = W.Workload("slabs", 16, 12, 8, 19, steps=4, ibnd=1, jbnd=0, kbnd=12, noise=3e-3, sphere=(6, 5, 4, 2))
NTILES = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def tile_start(wl, rank, ntiles):
    """The initialised global state (reference init order, FP32) cut to tile `rank`."""
    from oracle import oracle as O
    cfg = O.Config(wl.nx, wl.ny, wl.nz, wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=3, lsolids=True,
                   kinevisc=wl.kinevisc, smagorinsky=wl.smagorinsky)
    o = O.Oracle(cfg, np.float32)
    rho, u, v, w = W.initial_macro(wl)
    uvel = W.inflow_profile(wl)
    fA, fB = o.zeros_f(), o.zeros_f()
    o.init(fA, fB, rho, u, v, w, uvel)
    R = [o.zeros_s() for _ in range(4)]
    o.macrovars(*R, fA)
    cut = lambda a: np.ascontiguousarray(slabs.tile_slice(a, rank, ntiles))
    ny = wl.ny // ntiles
    tcfg = O.Config(wl.nx, ny, wl.nz, wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=3, lsolids=True,
                    kinevisc=wl.kinevisc, smagorinsky=wl.smagorinsky)
    t = dict(o=O.Oracle(tcfg, np.float32), f1=cut(fA), f2=cut(fB), R=[cut(a) for a in R],
             blank=cut(W.blanking(wl)).astype(np.int32), uvel=uvel, ny=ny,
             tau=np.full(tcfg.sshape, 3.0 * np.float32(wl.kinevisc) + 0.5, np.float32))
    return t


def collide_and_bound(t):
    t["o"].postcoll(t["f1"], t["tau"], *t["R"])
    t["o"].solids(t["f1"], t["blank"])
    t["o"].boundarycond(t["f1"], t["f2"], t["uvel"])


def stream(t):
    t["o"].drift(t["f2"], t["f1"])
    t["f1"], t["f2"] = t["f2"], t["f1"]
    t["o"].macrovars(*t["R"], t["f1"])


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method="env://")
    try:
        t = tile_start(WL, rank, world)
        ny = t["ny"]
        south, north = slabs.neighbours(rank, world, True)
        n = slabs.plane_bytes(WL.nx, WL.nz, WL.nl)
        plane_ok = True
        for _ in range(WL.steps):
            collide_and_bound(t)
            send_s = torch.from_numpy(slabs.plane_from_ref(t["f1"], 1))        # plane j = 1 goes south
            send_n = torch.from_numpy(slabs.plane_from_ref(t["f1"], ny))       # plane j = ny goes north
            assert send_s.numel() == n and send_n.numel() == n
            recv_s = torch.zeros(n, dtype=torch.uint8)
            recv_n = torch.zeros(n, dtype=torch.uint8)
            slabs.exchange(send_s, send_n, recv_s, recv_n, south, north)
            slabs.plane_to_ref(recv_s.numpy(), t["f1"], 0)
            slabs.plane_to_ref(recv_n.numpy(), t["f1"], ny + 1)
            # what arrived is what the neighbours packed: gather every rank's planes on every rank
            mine = torch.stack([send_s, send_n])
            allp = [torch.zeros_like(mine) for _ in range(world)]
            dist.all_gather(allp, mine)
            plane_ok &= bool(torch.equal(recv_s, allp[south][1]) and torch.equal(recv_n, allp[north][0]))
            stream(t)
        dist.barrier()
        out.put((rank, plane_ok, t["f1"], t["f2"], t["R"][0]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_exchange_lbm_planes():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, NTILES, port, q)) for r in range(NTILES)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(NTILES)), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # the same two tiles in one process, planes copied directly between the arrays
    tiles = [tile_start(WL, r, NTILES) for r in range(NTILES)]
    for _ in range(WL.steps):
        for t in tiles:
            collide_and_bound(t)
        planes = [(t["f1"][:, 1].copy(), t["f1"][:, t["ny"]].copy()) for t in tiles]
        for r, t in enumerate(tiles):
            south, north = slabs.neighbours(r, NTILES, True)
            t["f1"][:, 0] = planes[south][1]
            t["f1"][:, t["ny"] + 1] = planes[north][0]
        for t in tiles:
            stream(t)
    for (rank, plane_ok, f1, f2, rho), t in zip(res, tiles):
        assert plane_ok, "rank %d received planes other than its neighbours packed" % rank
        for name, a, b in (("f1", f1, t["f1"]), ("f2", f2, t["f2"]), ("rho", rho, t["R"][0])):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), "rank %d: %s" % (rank, name)


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_plane_codec_round_trip(storage):
    """plane_to_ref(plane_from_ref(f)) restores a near-equilibrium plane: exactly in
    FP32 (f - w_l is exact for f near w_l), to FP16 rounding of the 2^8-scaled
    offsets in FP16."""
    t = tile_start(WL, 0, NTILES)
    f = t["f1"]
    g = f.copy()
    b = slabs.plane_from_ref(f, 3, storage)
    assert b.size == slabs.plane_bytes(WL.nx, WL.nz, WL.nl, storage)
    g[:, 3] = 0
    slabs.plane_to_ref(b, g, 3, storage)
    if storage == "f32":
        assert np.array_equal(g, f)
    else:
        assert np.max(np.abs(g - f)) < 2e-5 and np.array_equal(np.delete(g, 3, 1), np.delete(f, 3, 1))
