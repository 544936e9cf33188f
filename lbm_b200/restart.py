"""Restart files of the reference (m_saverestart.F90:125-135, m_readrestart.F90:164-186).

``restart/restart_<tile>_<it>.uf`` holds one Fortran unformatted sequential
record ``nx, ny, nz, nl, f(nl,0:nx+1,0:ny+1,0:nz+1)``; f is the pre-collision
distribution f1 of step ``it`` (what the time loop holds after drift and the
pointer swap), ghost cells included.  On resume the reference reads f into fA,
recomputes rho, u, v, w with macrovars and copies fA to fB
(main.F90:255-259).

The record layout is the one gfortran writes: the record's bytes between a
leading and a trailing 4-byte length marker, split into subrecords of at most
2**31 - 9 bytes when longer.  A subrecord's leading marker is negative when
another subrecord follows, and its trailing marker is negative when another
precedes it.  Reading also accepts 8-byte markers (``-frecord-marker=8``).  f is
float32, or double precision in the reference's ``DP=1`` build: both are
written and read, and the reader converts to the precision the caller asks for.
"""
from __future__ import annotations

import os

import numpy as np

MAX_SUBRECORD = 2147483639


def restart_name(it: int, tile: int = 0, directory: str = "restart") -> str:
    """File name the reference uses for step ``it`` of MPI tile ``tile``."""
    return os.path.join(directory, "restart_%04d_%06d.uf" % (tile, it))


def write_record(fh, payload: bytes | memoryview, max_sub: int = MAX_SUBRECORD, marker: int = 4) -> None:
    """One Fortran unformatted sequential record."""
    mv = memoryview(payload).cast("B")
    n = len(mv)
    fmt = np.int32 if marker == 4 else np.int64
    chunks = [(o, min(max_sub, n - o)) for o in range(0, n, max_sub)] or [(0, 0)]
    for q, (o, m) in enumerate(chunks):
        more, prev = q + 1 < len(chunks), q > 0
        fh.write(np.array([-m if more else m], fmt).tobytes())
        fh.write(mv[o:o + m])
        fh.write(np.array([-m if prev else m], fmt).tobytes())


def _marker_size(fh) -> int:
    start = fh.tell()
    head = fh.read(8)
    fh.seek(start)
    if len(head) < 4:
        raise ValueError("not a Fortran unformatted record: file too short")
    for size, fmt in ((4, "<i4"), (8, "<i8")):
        m = abs(int(np.frombuffer(head[:size], fmt)[0]))
        fh.seek(start + size + m)
        tail = fh.read(size)
        fh.seek(start)
        if len(tail) == size and abs(int(np.frombuffer(tail, fmt)[0])) == m:
            return size
    raise ValueError("not a Fortran unformatted record: markers do not match")


def read_record(fh) -> bytes:
    """The payload of the next record (subrecords joined)."""
    size = _marker_size(fh)
    fmt = "<i4" if size == 4 else "<i8"
    parts = []
    while True:
        lead = int(np.frombuffer(fh.read(size), fmt)[0])
        n = abs(lead)
        data = fh.read(n)
        trail = fh.read(size)
        if len(data) != n or len(trail) != size or abs(int(np.frombuffer(trail, fmt)[0])) != n:
            raise ValueError("truncated or corrupt Fortran record")
        parts.append(data)
        if lead >= 0:
            return b"".join(parts)


def write_restart(path: str, f, nx: int, ny: int, nz: int, nl: int, max_sub: int = MAX_SUBRECORD,
                  dtype=np.float32) -> None:
    """Write f (reference layout, C order (nz+2, ny+2, nx+2, nl)) as the reference does:
    float32, or dtype=np.float64 for the record of its DP build (real(8) f)."""
    if np.dtype(dtype) not in (np.dtype(np.float32), np.dtype(np.float64)):
        raise ValueError("restart payloads are float32 or float64, not %s" % np.dtype(dtype))
    a = np.ascontiguousarray(np.asarray(f, dtype=dtype))
    if a.shape != (nz + 2, ny + 2, nx + 2, nl):
        raise ValueError("f has shape %s, expected %s" % (a.shape, (nz + 2, ny + 2, nx + 2, nl)))
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    head = np.array([nx, ny, nz, nl], np.int32).tobytes()
    payload = bytearray(len(head) + a.nbytes)
    payload[:len(head)] = head
    payload[len(head):] = a.tobytes()
    with open(path, "wb") as fh:
        write_record(fh, payload, max_sub)


def read_restart(path: str, expect=None, dtype=np.float32):
    """(nx, ny, nz, nl, f in C order (nz+2, ny+2, nx+2, nl)) with f converted to
    ``dtype`` (float32 for the fused state and the FP32 entry points, float64 for
    the _f64 ones; either record precision is read).  With ``expect`` = (nx, ny,
    nz, nl), other dimensions raise ValueError (the reference stops)."""
    with open(path, "rb") as fh:
        rec = read_record(fh)
    nx, ny, nz, nl = (int(x) for x in np.frombuffer(rec[:16], "<i4"))
    if expect is not None and (nx, ny, nz, nl) != tuple(expect):
        raise ValueError("restart file %s has dimensions %s, expected %s" % (path, (nx, ny, nz, nl), tuple(expect)))
    n = (nx + 2) * (ny + 2) * (nz + 2) * nl
    body = len(rec) - 16
    if body == 4 * n:
        f = np.frombuffer(rec, "<f4", count=n, offset=16)
    elif body == 8 * n:
        f = np.frombuffer(rec, "<f8", count=n, offset=16)
    else:
        raise ValueError("restart record of %d bytes does not hold f for %s" % (len(rec), (nx, ny, nz, nl)))
    return nx, ny, nz, nl, f.astype(dtype).reshape(nz + 2, ny + 2, nx + 2, nl)


def save_state(lbm, path: str) -> None:
    """saverestart of a fused state: the reference's f1 of the current step."""
    import torch
    f1, f2 = lbm.empty_f(), lbm.empty_f()
    lbm.state_export(f1, f2)
    torch.cuda.synchronize()
    p = lbm.p
    write_restart(path, f1.cpu().numpy(), p.nx, p.ny, p.nz, p.nl)


def load_state(lbm, path: str, it: int) -> None:
    """readrestart into a context: f1 from the file, rho, u, v, w = macrovars(f1),
    f2 = f1 (main.F90:255-259), imported as the state after step ``it``."""
    import torch
    p = lbm.p
    *_, f = read_restart(path, expect=(p.nx, p.ny, p.nz, p.nl))
    f1 = torch.from_numpy(f).cuda()
    rho, u, v, w = (lbm.empty_s() for _ in range(4))
    lbm.macrovars(rho, u, v, w, f1)
    lbm.state_import(f1, f1.clone(), rho, u, v, w, it=it)
