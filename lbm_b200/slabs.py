"""One domain split into j slabs, one tile per context (or per GPU), as the
reference's MPI tiling does (m_mpi_decomp_init.F90:93-134,
m_mpi_halo_exchange_j.F90:3-121, m_mpi_pack_jplane.F90, m_mpi_unpack_jplane.F90).

The global interior rows 1..nyg are cut into ntiles tiles of ny = nyg / ntiles
rows; tile r holds global rows r*ny+1 .. (r+1)*ny and stores ghost planes
j = 0 and ny+1.  A tile steps with its own boundary conditions (the
reference's boundarycond, tile by tile), then exchanges its halo: plane j = ny
goes north into the neighbour's j = 0, plane j = 1 goes south into the
neighbour's j = ny+1.  With periodic j the tiles form a ring; otherwise the end
tiles have no neighbour on the open side and keep their own boundary values.

The exchange is two shifts, north then south, each posted as one batch of
point-to-point operations (NCCL over NVLink between GPUs, gloo on the host).
Every rank posts them in the same order, so the messages between a pair of
ranks match even when that pair is both neighbours of each other (two tiles in
a ring).
"""
from __future__ import annotations

import torch

from .api import Lbm, Params


def tile_rows(nyg: int, ntiles: int, rank: int) -> tuple[int, int]:
    """(first global row, rows) of tile ``rank``; the reference stops unless
    ntiles divides nyg (m_mpi_decomp_init.F90:93-96)."""
    if ntiles < 1 or not 0 <= rank < ntiles:
        raise ValueError("rank %d of %d tiles" % (rank, ntiles))
    if nyg % ntiles != 0:
        raise ValueError("nyg = %d is not a multiple of the %d tiles" % (nyg, ntiles))
    ny = nyg // ntiles
    return rank * ny + 1, ny


def neighbours(rank: int, ntiles: int, periodic: bool) -> tuple[int | None, int | None]:
    """(south, north) ranks of tile ``rank`` (m_mpi_decomp_init.F90:128-134);
    None where a non-periodic domain ends."""
    if periodic:
        return (rank - 1) % ntiles, (rank + 1) % ntiles
    return (rank - 1 if rank > 0 else None), (rank + 1 if rank + 1 < ntiles else None)


def tile_slice(a, rank: int, ntiles: int):
    """The rows of tile ``rank`` (with its two ghost rows) of a global array in
    the reference layout, C order (nz+2, nyg+2, nx+2[, nl])."""
    j0, ny = tile_rows(a.shape[1] - 2, ntiles, rank)
    return a[:, j0 - 1:j0 + ny + 1]


def plane_bytes(nx: int, nz: int, nl: int, storage: str = "f32") -> int:
    """Bytes of one packed halo plane, as lbm_halo_plane_bytes reports them:
    nl x (nz+2) x (nx+2) state values of 4 (FP32) or 2 (FP16) bytes."""
    return nl * (nz + 2) * (nx + 2) * (2 if storage == "f16" else 4)


def _weights(nl: int):
    import numpy as np
    c = np.array([[0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1],
                  [0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 0, 0, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1],
                  [0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1]])[:, :nl]
    s2 = (c * c).sum(0)
    tab = {19: (1 / 3, 1 / 18, 1 / 36, 0.0), 27: (8 / 27, 2 / 27, 1 / 54, 1 / 216)}[nl]
    return np.array([tab[k] for k in s2], dtype=np.float32)


def plane_from_ref(f, j: int, storage: str = "f32"):
    """Host mirror of lbm_halo_pack_j's plane layout: the bytes of plane j of a
    reference-layout array f (nz+2, ny+2, nx+2, nl) as the state stores it,
    values[l][k][i] (i = 0..nx+1 fastest) of the offset f - w_l, in FP32 or as
    FP16 of (f - w_l) * 2^8."""
    import numpy as np
    nl = f.shape[-1]
    off = (f[:, j].astype(np.float32) - _weights(nl)).transpose(2, 0, 1)      # (nl, nz+2, nx+2)
    if storage == "f16":
        return np.ascontiguousarray((off * np.float32(256.0)).astype(np.float16)).view(np.uint8).ravel()
    return np.ascontiguousarray(off, dtype=np.float32).view(np.uint8).ravel()


def plane_to_ref(buf, f, j: int, storage: str = "f32"):
    """Inverse of plane_from_ref: write a packed plane into plane j of f."""
    import numpy as np
    nl = f.shape[-1]
    nzp, nxp = f.shape[0], f.shape[2]
    b = np.ascontiguousarray(buf, dtype=np.uint8)
    if storage == "f16":
        off = b.view(np.float16).astype(np.float32) / np.float32(256.0)
    else:
        off = b.view(np.float32)
    f[:, j] = (off.reshape(nl, nzp, nxp).transpose(1, 2, 0) + _weights(nl)).astype(f.dtype)


def exchange(send_south, send_north, recv_south, recv_north, south, north, group=None):
    """The halo exchange of one rank through torch.distributed: send_north goes
    to ``north`` and arrives there as its recv_south; send_south goes to
    ``south`` and arrives there as its recv_north.  A neighbour of None is
    skipped.  Shift north first, then south."""
    import torch.distributed as dist
    for dst, src, send, recv in ((north, south, send_north, recv_south), (south, north, send_south, recv_north)):
        ops = []
        if src is not None:
            ops.append(dist.P2POp(dist.irecv, recv, src, group))
        if dst is not None:
            ops.append(dist.P2POp(dist.isend, send, dst, group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()


class SlabTile:
    """One tile: a context of ny = nyg / ntiles rows with stored j ghost planes
    (lbm_set_halo_j) and its plane buffers."""

    def __init__(self, params: Params, rank: int, ntiles: int, periodic: bool | None = None, stream=None):
        self.gp = params
        self.rank, self.ntiles = rank, ntiles
        self.j0, ny = tile_rows(params.ny, ntiles, rank)
        self.periodic = (params.jbnd == 0) if periodic is None else periodic
        self.south, self.north = neighbours(rank, ntiles, self.periodic)
        import dataclasses
        self.p = dataclasses.replace(params, ny=ny)
        self.lbm = Lbm(self.p, stream=stream)
        self.lbm.set_halo_j(True)
        n = self.lbm.halo_plane_bytes()
        self.send = [torch.empty(n, dtype=torch.uint8, device="cuda") for _ in range(2)]   # to south, to north
        self.recv = [torch.empty(n, dtype=torch.uint8, device="cuda") for _ in range(2)]   # from south, from north

    def import_global(self, f1, f2, rho, u, v, w, it: int = 0):
        """Import the tile's rows of a global state (reference layout, device)."""
        cut = [tile_slice(a, self.rank, self.ntiles).contiguous() for a in (f1, f2, rho, u, v, w)]
        self.lbm.state_import(*cut, it=it)

    def set_solids(self, blanking):
        self.lbm.set_solids(tile_slice(blanking, self.rank, self.ntiles).contiguous())

    def set_inflow(self, uvel):
        self.lbm.set_inflow(uvel)

    def pack(self):
        self.lbm.halo_pack_j(self.send[0] if self.south is not None else None,
                             self.send[1] if self.north is not None else None)

    def unpack(self):
        self.lbm.halo_unpack_j(self.recv[0] if self.south is not None else None,
                               self.recv[1] if self.north is not None else None)

    def step(self, n: int = 1, group=None):
        """n steps of this rank's tile with a halo exchange after each (one
        tile per rank of the default or given process group)."""
        cur = torch.cuda.current_stream()
        for _ in range(n):
            self.lbm.step(1)
            self.pack()
            cur.wait_stream(self.lbm.stream)          # the sends read the packed planes
            exchange(self.send[0], self.send[1], self.recv[0], self.recv[1], self.south, self.north, group)
            self.lbm.stream.wait_stream(cur)          # the unpack reads what arrived
            self.unpack()

    def close(self):
        self.lbm.close()


def step_local(tiles: list[SlabTile], n: int = 1):
    """n steps of all tiles of a domain held in one process (one device): each
    tile steps, then the planes move between the tiles' buffers."""
    cur = torch.cuda.current_stream()
    for _ in range(n):
        for t in tiles:
            t.lbm.step(1)
            t.pack()
        for t in tiles:
            cur.wait_stream(t.lbm.stream)
        for t in tiles:
            if t.south is not None:
                t.recv[0].copy_(tiles[t.south].send[1])
            if t.north is not None:
                t.recv[1].copy_(tiles[t.north].send[0])
        for t in tiles:
            t.lbm.stream.wait_stream(cur)
            t.unpack()
