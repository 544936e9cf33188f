"""Restart files in the reference's Fortran unformatted layout (no GPU)."""
import io

import numpy as np
import pytest

from lbm_b200 import restart as R


def test_single_record_bytes(tmp_path):
    nx, ny, nz, nl = 2, 1, 1, 19
    f = np.arange((nz + 2) * (ny + 2) * (nx + 2) * nl, dtype=np.float32).reshape(nz + 2, ny + 2, nx + 2, nl)
    p = tmp_path / "restart_0000_000007.uf"
    R.write_restart(str(p), f, nx, ny, nz, nl)
    raw = p.read_bytes()
    n = 16 + f.nbytes
    assert len(raw) == n + 8
    assert np.frombuffer(raw[:4], "<i4")[0] == n and np.frombuffer(raw[-4:], "<i4")[0] == n
    assert list(np.frombuffer(raw[4:20], "<i4")) == [nx, ny, nz, nl]
    # column-major f(nl,0:nx+1,0:ny+1,0:nz+1): l fastest, then i, j, k
    assert np.array_equal(np.frombuffer(raw[20:-4], "<f4"), f.ravel())
    out = R.read_restart(str(p), expect=(nx, ny, nz, nl))
    assert out[:4] == (nx, ny, nz, nl) and np.array_equal(out[4], f)


def test_subrecords_follow_the_sign_convention():
    payload = bytes(range(200)) * 2                      # 400 bytes in subrecords of at most 150
    fh = io.BytesIO()
    R.write_record(fh, payload, max_sub=150)
    raw = fh.getvalue()
    marks = []
    pos = 0
    while pos < len(raw):
        lead = int(np.frombuffer(raw[pos:pos + 4], "<i4")[0])
        n = abs(lead)
        trail = int(np.frombuffer(raw[pos + 4 + n:pos + 8 + n], "<i4")[0])
        marks.append((lead, trail))
        pos += n + 8
    # first: more follow (lead < 0), none before (trail > 0); middle: both negative; last: lead > 0, trail < 0
    assert marks == [(-150, 150), (-150, -150), (100, -100)]
    fh.seek(0)
    assert R.read_record(fh) == payload


def test_eight_byte_markers_and_double_precision(tmp_path):
    nx, ny, nz, nl = 3, 2, 2, 19
    f64 = np.random.default_rng(1).standard_normal((nz + 2, ny + 2, nx + 2, nl))
    p = tmp_path / "dp.uf"
    with open(p, "wb") as fh:
        R.write_record(fh, np.array([nx, ny, nz, nl], np.int32).tobytes() + f64.tobytes(), marker=8)
    out = R.read_restart(str(p))
    assert out[:4] == (nx, ny, nz, nl)
    assert np.array_equal(out[4], f64.astype(np.float32))


def test_double_precision_record_round_trip(tmp_path):
    """The DP build's record (real(8) f) as written here: 8 bytes per value between
    the markers, read back bit for bit as float64 and rounded once as float32."""
    nx, ny, nz, nl = 3, 2, 2, 27
    f64 = np.random.default_rng(2).standard_normal((nz + 2, ny + 2, nx + 2, nl))
    p = tmp_path / "restart_0000_000003.uf"
    R.write_restart(str(p), f64, nx, ny, nz, nl, dtype=np.float64)
    raw = p.read_bytes()
    n = 16 + f64.nbytes
    assert len(raw) == n + 8 and np.frombuffer(raw[:4], "<i4")[0] == n
    assert np.array_equal(np.frombuffer(raw[20:-4], "<f8"), f64.ravel())
    out = R.read_restart(str(p), expect=(nx, ny, nz, nl), dtype=np.float64)
    assert out[4].dtype == np.float64 and np.array_equal(out[4], f64)
    assert np.array_equal(R.read_restart(str(p))[4], f64.astype(np.float32))
    with pytest.raises(ValueError):
        R.write_restart(str(p), f64, nx, ny, nz, nl, dtype=np.float16)


def test_dimension_mismatch_and_corruption(tmp_path):
    nx, ny, nz, nl = 2, 2, 2, 27
    f = np.zeros((nz + 2, ny + 2, nx + 2, nl), np.float32)
    p = tmp_path / "r.uf"
    R.write_restart(str(p), f, nx, ny, nz, nl)
    with pytest.raises(ValueError, match="dimensions"):
        R.read_restart(str(p), expect=(nx, ny, nz, 19))
    raw = p.read_bytes()
    (tmp_path / "cut.uf").write_bytes(raw[:-10])
    with pytest.raises(ValueError):
        R.read_restart(str(tmp_path / "cut.uf"))
    with pytest.raises(ValueError, match="shape"):
        R.write_restart(str(p), f[:, :, :, :19], nx, ny, nz, nl)


def test_file_name_convention():
    assert R.restart_name(1000) == "restart/restart_0000_001000.uf"
    assert R.restart_name(7, tile=3, directory="out") == "out/restart_0003_000007.uf"
