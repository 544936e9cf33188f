"""The allocation-free conservation entry point, through the C ABI.

lbm_mass_momentum_noalloc serves callers that cannot allocate device memory
(their device memory belongs to another runtime's pool, or a cudaMalloc inside
their loop would synchronise the device).  It must give the same FP64 sums as
the context-based lbm_mass_momentum, call after call, while keeping its
partial sums in the library's fixed device array.  This file is collected last
so that a run stopping at the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")


@pytest.mark.gpu
def test_noalloc_sums_match_context_sums_on_consecutive_calls():
    from lbm_b200 import Lbm, Params, _lib
    nx, ny, nz, nl = 96, 40, 24, 27
    L = Lbm(Params(nx=nx, ny=ny, nz=nz, nl=nl, iturb_pos=3))
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(21)
    for call in range(2):
        f = torch.from_numpy(rng.uniform(0.0, 0.1, L.p.fshape).astype(np.float32)).cuda()
        ref = L.mass_momentum(f)
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.lbm_mass_momentum_noalloc(ctypes.c_void_p(f.data_ptr()), nx, ny, nz, nl,
                                           ctypes.c_void_p(out.data_ptr()), stream)
        assert rc == 0, "call %d returned %d" % (call, rc)
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=1e-12, atol=1e-9)
    # a grid above the fixed scratch capacity is refused before any device work
    rc = lib.lbm_mass_momentum_noalloc(ctypes.c_void_p(f.data_ptr()), 1024, 1024, 1024, nl,
                                       ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == _lib.LBM_ERR_ARG


def _fp64_sums(f, nl, chunk=16):
    """mass and momentum of the interior cells in FP64, summed on the device by k slabs"""
    from oracle import oracle as O
    t = O.tables(nl, np.float64)
    c = torch.tensor(np.stack([np.ones(nl), t["cx"], t["cy"], t["cz"]]), dtype=torch.float64, device=f.device)
    per_l = torch.zeros(nl, dtype=torch.float64, device=f.device)
    nz = f.shape[0] - 2
    for k0 in range(1, nz + 1, chunk):
        k1 = min(nz + 1, k0 + chunk)
        per_l += f[k0:k1, 1:-1, 1:-1, :].double().sum(dim=(0, 1, 2))
    return (c @ per_l).cpu().numpy()


@pytest.mark.gpu
def test_noalloc_sums_near_the_cell_cap():
    """A grid just below the 134,217,728-cell cap (2,032 block partials, so the final
    sum walks far more partials than it has threads), twice in a row, against FP64
    sums of the same array."""
    from lbm_b200 import _lib
    nx, ny, nz, nl = 1024, 512, 254, 19
    assert nx * ny * nz <= 2048 * 65536 and nx * ny * nz > 2000 * 65536
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    f = torch.rand((nz + 2, ny + 2, nx + 2, nl), generator=gen, device="cuda", dtype=torch.float32) * 0.1
    ref = _fp64_sums(f, nl)
    for call in range(2):
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.lbm_mass_momentum_noalloc(ctypes.c_void_p(f.data_ptr()), nx, ny, nz, nl,
                                           ctypes.c_void_p(out.data_ptr()), stream)
        assert rc == 0, "call %d returned %d" % (call, rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got[0], ref[0], rtol=1e-12)
        np.testing.assert_allclose(got[1:], ref[1:], rtol=1e-12, atol=1e-12 * ref[0])
    del f
    torch.cuda.empty_cache()
