"""FP64 mass/momentum reductions (per-call and fused state) through the C ABI."""
import numpy as np
import pytest

from lbm_b200 import workloads as W

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def ref_sums(f, nl):
    from oracle import oracle as O
    t = O.tables(nl, np.float64)
    c = np.stack([t["cx"], t["cy"], t["cz"]], 1).astype(np.float64)
    fi = f[1:-1, 1:-1, 1:-1].astype(np.float64)
    return np.array([fi.sum(), *(fi @ c).sum(axis=(0, 1, 2))])


@pytest.mark.parametrize("nl", [19, 27])
def test_mass_momentum_reference_layout(nl):
    from lbm_b200 import Lbm, Params
    L = Lbm(Params(nx=37, ny=21, nz=13, nl=nl, iturb_pos=3))
    rng = np.random.default_rng(4)
    f = rng.uniform(0.0, 0.1, L.p.fshape).astype(np.float32)
    out = L.mass_momentum(torch.from_numpy(f).cuda()).cpu().numpy()
    ref = ref_sums(f, nl)
    # every population enters in FP64: only the order of the FP64 additions differs
    np.testing.assert_allclose(out[0], ref[0], rtol=1e-12)
    np.testing.assert_allclose(out[1:], ref[1:], rtol=1e-12, atol=1e-12 * abs(ref[0]))


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_periodic_box_conserves_mass_and_momentum(storage):
    from lbm_b200 import Lbm, Params
    nx, ny, nz = 64, 32, 24
    L = Lbm(Params(nx=nx, ny=ny, nz=nz, nl=27, ibnd=0, jbnd=0, kbnd=0, storage=storage))
    wl = W.Workload("box", nx, ny, nz, 27, noise=2e-2, ibnd=0, jbnd=0, kbnd=0)
    rho, u, v, w = (torch.from_numpy(a).cuda() for a in W.initial_macro(wl))
    f1 = L.empty_f()
    L.fequil3(f1, rho, u, v, w)
    L.fillghosts(f1)
    f2 = f1.clone()
    L.boundarycond(f1, f2, None)
    L.state_import(f1, f2, rho, u, v, w)
    m0 = np.array(L.conservation())
    ref0 = ref_sums(f1.cpu().numpy(), 27)
    # FP16 storage quantizes the imported offsets (~1e-3 of each, sign-random)
    np.testing.assert_allclose(m0, ref0, rtol=2e-7, atol=1e-6 if storage == "f32" else 1e-3)
    L.step(20)
    m1 = np.array(L.conservation())
    tol = 1e-7 if storage == "f32" else 1e-4
    assert abs(m1[0] - m0[0]) <= tol * m0[0], (m0, m1)
    np.testing.assert_allclose(m1[1:], m0[1:], atol=tol * m0[0])
    # the fused-state sum equals the sum of the exported reference-layout f1
    e1, e2 = L.empty_f(), L.empty_f()
    L.state_export(e1, e2)
    np.testing.assert_allclose(L.mass_momentum(e1).cpu().numpy(), m1, rtol=1e-6, atol=1e-6)
