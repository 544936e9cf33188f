"""States of more than 2^31 elements per buffer: every offset of the step is
64-bit.  A domain periodic in j is invariant under shifts in j, so a domain
made of M copies of a small one along j (state, solids and turbulence slice
alike) evolves into M copies of the small domain's result, bit for bit: each
cell of the large run does the arithmetic of its counterpart in the small run,
which the other GPU tests check against the oracle.  The large domain is
128 x 6720 x 62 (53 M cells): 27 x 82.6 M elements per D3Q27 state buffer."""
import numpy as np
import pytest

from lbm_b200 import workloads as W
from tests.test_gpu_fused import cuda, params_of
from tests.test_gpu_slabs import global_start

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

NY_SMALL, COPIES = 16, 420


def tile_j(a, m, axis=1):
    """A reference-layout array (C order (nz+2, ny+2, nx+2[, nl])) of the small
    domain repeated m times along the interior rows; its ghost rows stay."""
    shape = list(a.shape)
    shape[axis] = (shape[axis] - 2) * m + 2
    out = torch.empty(shape, dtype=a.dtype, device=a.device)
    lo = [slice(None)] * a.dim()
    hi = [slice(None)] * a.dim()
    lo[axis], hi[axis] = 0, -1
    out[tuple(lo)] = a[tuple(lo)]
    out[tuple(hi)] = a[tuple(hi)]
    inner = [slice(None)] * a.dim()
    inner[axis] = slice(1, -1)
    src = a[tuple(inner)].unsqueeze(axis)
    dst_shape = list(src.shape)
    dst_shape[axis] = m
    out[tuple(inner)].view(*shape[:axis], m, a.shape[axis] - 2, *shape[axis + 1:]).copy_(src.expand(dst_shape))
    return out


def prepare(L, state, blank, uvel, turb):
    if blank is not None:
        L.set_solids(blank)
    L.set_inflow(uvel)
    if turb is not None:
        L.set_turbulence(*turb, nrturb=turb[0].shape[0] - 1, ampl=1.0e-3)
    L.state_import(*state)


def result(L):
    f1, f2 = L.empty_f(), L.empty_f()
    L.state_export(f1, f2)
    m = [L.empty_s() for _ in range(4)]
    L.get_macro(*m)
    torch.cuda.synchronize()
    return [f1, f2, *m], L.status()


def run(p, state, blank, uvel, turb, steps):
    from lbm_b200 import Lbm
    L = Lbm(p)
    prepare(L, state, blank, uvel, turb)
    L.step(steps)
    out = result(L)
    L.close()
    return out


def same_bits(big, small, m):
    """big (ny = m * ny_small) equals small tiled m times along j, bit for bit."""
    if not torch.equal(big[:, 0].view(torch.int32), small[:, 0].view(torch.int32)):
        return False
    if not torch.equal(big[:, -1].view(torch.int32), small[:, -1].view(torch.int32)):
        return False
    inner = big[:, 1:-1]
    tiles = inner.reshape(inner.shape[0], m, small.shape[1] - 2, *inner.shape[2:])
    return bool(torch.equal(tiles.view(torch.int32), small[:, 1:-1].unsqueeze(1).expand_as(tiles).view(torch.int32)))


@pytest.mark.parametrize("codes,storage,turbulence,ensemble", [((1, 0, 12), "f32", True, True),
                                                              ((1, 0, 12), "f16", True, False),
                                                              ((0, 0, 0), "f32", False, False)])
def test_state_past_2_to_31_elements(codes, storage, turbulence, ensemble):
    """ensemble: the small and the large domain also run as the two members of
    one batched ensemble, which must reproduce their separate runs bit for bit."""
    ib, jb, kb = codes
    wl = W.Workload("large", 128, NY_SMALL, 62, 27, steps=6, ibnd=ib, jbnd=jb, kbnd=kb, noise=3e-3,
                    sphere=(40, 8, 20, 5))
    fA, fB, R, blank, uvel = global_start(wl)
    small_state = [cuda(a.astype(np.float32)) for a in (fA, fB, *R)]
    blank_s = cuda(blank.astype(np.int32))
    uvel_d = cuda(uvel.astype(np.float32))
    turb_s = None
    if turbulence:
        rng = np.random.default_rng(5)
        turb_s = [cuda(rng.standard_normal((9, wl.nz, wl.ny)).astype(np.float32)) for _ in range(3)]
    p_small = params_of(wl, iturb_pos=3, storage=storage)
    small, st_small = run(p_small, small_state, blank_s, uvel_d, turb_s, wl.steps)

    big_wl = wl.with_(ny=NY_SMALL * COPIES)
    p_big = params_of(big_wl, iturb_pos=3, storage=storage)
    pitch = ((big_wl.nx + 34 + 31) // 32) * 32
    assert 27 * (big_wl.ny + 2) * (big_wl.nz + 2) * pitch > 2 ** 31
    big_state = [tile_j(a, COPIES) for a in small_state]
    turb_b = None
    if turbulence:
        turb_b = [t.repeat(1, 1, COPIES) for t in turb_s]
    blank_b = tile_j(blank_s, COPIES)
    big, st_big = run(p_big, big_state, blank_b, uvel_d, turb_b, wl.steps)
    assert st_small == 0 and st_big == 0
    assert torch.isfinite(small[0]).all()
    for name, b, s in zip(("f1", "f2", "rho", "u", "v", "w"), big, small):
        assert same_bits(b, s, COPIES), name
    if ensemble:
        from lbm_b200 import Ensemble
        ens = Ensemble([p_small, p_big])
        prepare(ens.members[0], small_state, blank_s, uvel_d, turb_s)
        prepare(ens.members[1], big_state, blank_b, uvel_d, turb_b)
        del big_state
        ens.step(wl.steps)
        for alone, L in ((small, ens.members[0]), (big, ens.members[1])):
            batched, st = result(L)
            assert st == 0
            for name, a, b in zip(("f1", "f2", "rho", "u", "v", "w"), batched, alone):
                assert torch.equal(a.view(torch.int32), b.view(torch.int32)), "ensemble " + name
            del batched
        ens.close()
