"""Per-call entry points (reference interfaces) vs the oracle, through the C ABI.

Copies and permutations (drift, boundary copies, solids, fillghosts,
compute_f/fneq, turbulence apply) must match the FP32 oracle bit for bit;
macrovars keeps the reference's summation order and matches bit for bit too.
Floating-point collision routines are evaluated in closed form and must stay
within FP32 round-off of the oracle: relative L2 <= 2e-6 against the FP64
oracle, the FP32 oracle's own distance being of the same order."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

NX, NY, NZ = 4, 3, 3


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def mk(nl, **kw):
    from lbm_b200 import Lbm, Params
    base = dict(nx=NX, ny=NY, nz=NZ, nl=nl, iturb_pos=3)
    base.update(kw)
    return Lbm(Params(**base))


def ocfg(nl, **kw):
    base = dict(nx=NX, ny=NY, nz=NZ, nl=nl, iturb_pos=3, nrturb=4, ampl=1e-2)
    base.update(kw)
    return O.Config(**base)


def g32(golden, name):
    return np.ascontiguousarray(golden[name].astype(np.float32))


@pytest.fixture(params=[19, 27])
def nl(request):
    return request.param


def test_fequil3(golden, nl):
    p = "q%d_" % nl
    for ibgk, key in ((3, "fequil3"), (2, "fequil2")):
        L = mk(nl, ibgk=ibgk)
        feq = L.empty_f()
        L.fequil3(feq, *(dev(g32(golden, p + n)) for n in ("rho", "u", "v", "w")))
        out = host(feq)
        s = (slice(1, -1),) * 3
        assert rel_l2(out[s], golden[p + key][s]) < 2e-7
        assert np.all(out[0] == 0) and np.all(out[:, 0] == 0)   # ghosts untouched


@pytest.mark.parametrize("ihrr", [0, 1])
@pytest.mark.parametrize("ivr", [0, 1])
def test_postcoll(golden, nl, ihrr, ivr):
    p = "q%d_" % nl
    L = mk(nl, ihrr=ihrr, ivreman=ivr)
    f = dev(g32(golden, p + "f"))
    tau = dev(np.full((NZ + 2, NY + 2, NX + 2), 3 * np.float32(1e-4) + 0.5, np.float32))
    L.postcoll(f, tau, *(dev(g32(golden, p + n)) for n in ("rho", "u", "v", "w")))
    fo, to = host(f), host(tau)
    s = (slice(1, -1),) * 3
    ref_f = golden[p + "postcoll_h%d_v%d_f" % (ihrr, ivr)]
    ref_t = golden[p + "postcoll_h%d_v%d_tau" % (ihrr, ivr)]
    assert rel_l2(fo[s], ref_f[s]) < 2e-6
    # the eddy viscosity is a small difference of squares: FP32 keeps ~1e-4 of it
    assert rel_l2(to[s] - 0.5, ref_t[s] - 0.5) < 2e-4
    np.testing.assert_array_equal(fo[0], g32(golden, p + "f")[0])    # ghosts untouched


def test_drift_bitexact(golden, nl):
    p = "q%d_" % nl
    L = mk(nl)
    fin = dev(g32(golden, p + "f"))
    fout = L.empty_f()
    L.drift(fout, fin)
    o = O.Oracle(ocfg(nl), np.float32)
    ref = o.zeros_f()
    o.drift(ref, g32(golden, p + "f"))
    np.testing.assert_array_equal(host(fout), ref)


def test_macrovars_bitexact(golden, nl):
    p = "q%d_" % nl
    L = mk(nl)
    out = [L.empty_s() for _ in range(4)]
    L.macrovars(*out, dev(g32(golden, p + "f")))
    o = O.Oracle(ocfg(nl), np.float32)
    ref = [o.zeros_s() for _ in range(4)]
    o.macrovars(*ref, g32(golden, p + "f"))
    for a, b in zip(out, ref):
        np.testing.assert_array_equal(host(a), b)


def test_regularization_and_vreman(golden, nl):
    p = "q%d_" % nl
    L = mk(nl)
    f = dev(g32(golden, p + "f"))
    L.regularization(f, dev(g32(golden, p + "fequil3")), *(dev(g32(golden, p + n)) for n in ("u", "v", "w")))
    s = (slice(1, -1),) * 3
    assert rel_l2(host(f)[s], golden[p + "regularization"][s]) < 2e-5
    tau = L.empty_s()
    L.vreman(dev(g32(golden, p + "vreman_in")), tau)
    assert rel_l2(host(tau)[s] - 0.5, golden[p + "vreman_tau"][s] - 0.5) < 1e-4


def test_compute_f_and_fneq_bitexact(golden, nl):
    p = "q%d_" % nl
    L = mk(nl)
    a, b = g32(golden, p + "f"), g32(golden, p + "fequil3")
    f = dev(a)
    L.compute_fneq(f, dev(b))
    np.testing.assert_array_equal(host(f), a - b)
    L.compute_f(f, dev(b))
    np.testing.assert_array_equal(host(f), b + (a - b))


@pytest.mark.parametrize("codes", [(1, 0, 12), (0, 0, 0), (11, 22, 12), (22, 21, 11), (12, 11, 22), (1, 11, 22)])
def test_boundarycond(golden, nl, codes):
    p = "q%d_" % nl
    ib, jb, kb = codes
    udir = 10.0 if ib == 1 else 0.0
    L = mk(nl, ibnd=ib, jbnd=jb, kbnd=kb, udir=udir)
    f1, f2 = g32(golden, p + "bc_f1"), g32(golden, p + "bc_f2")
    uvel = g32(golden, p + "bc_uvel")
    d1, d2 = dev(f1), dev(f2)
    L.boundarycond(d1, d2, dev(uvel))
    o = O.Oracle(ocfg(nl, ibnd=ib, jbnd=jb, kbnd=kb, udir=udir), np.float32)
    r1, r2 = f1.copy(), f2.copy()
    o.boundarycond(r1, r2, uvel)
    out = host(d1)
    if ib == 1:
        np.testing.assert_array_equal(out[:, :, 1:], r1[:, :, 1:])
        assert rel_l2(out, r1) < 1e-7
    else:
        np.testing.assert_array_equal(out, r1)
    np.testing.assert_array_equal(host(d2), f2)


def test_solids_fillghosts_bitexact(golden, nl):
    p = "q%d_" % nl
    L = mk(nl)
    f = dev(g32(golden, p + "f"))
    L.solids(f, dev(golden[p + "solids_mask"].astype(np.int32)))
    np.testing.assert_array_equal(host(f), golden[p + "solids"].astype(np.float32))
    f = dev(g32(golden, p + "f"))
    L.fillghosts(f)
    np.testing.assert_array_equal(host(f), golden[p + "fillghosts"].astype(np.float32))


def test_turbulence_forcing_and_apply(golden, nl):
    p = "q%d_" % nl
    L = mk(nl)
    df = torch.zeros((NZ, NY, nl), dtype=torch.float32, device="cuda")
    uu, vv, ww = (dev(g32(golden, p + n)) for n in ("turb_uu", "turb_vv", "turb_ww"))
    L.inflow_turbulence_forcing(df, *(dev(g32(golden, p + n)) for n in ("rho", "u", "v", "w")), uu, vv, ww,
                                1e-2, 7, 4)
    out = host(df)
    # the FP64 restatement is the yardstick: the difference of equilibria is formed analytically here
    assert rel_l2(out, golden[p + "turb_df_it7"]) < 5e-6
    f = dev(g32(golden, p + "f"))
    L.inflow_turbulence_apply(f, df)
    o = O.Oracle(ocfg(nl), np.float32)
    ref = g32(golden, p + "f")
    o.turbulence_apply(ref, out)
    np.testing.assert_array_equal(host(f), ref)


def test_argument_errors(nl):
    from lbm_b200 import LbmError
    L = mk(nl)
    with pytest.raises(LbmError):
        L.drift(L.empty_f()[:, :, :, :-1].contiguous(), L.empty_f())      # wrong shape
    f = L.empty_f()
    with pytest.raises(LbmError):
        L.drift(f, f)                                                       # aliasing
    with pytest.raises(LbmError):
        L.step(1)                                                           # no state imported


# ---- the DP build's entry points (_f64): float64 arrays against the FP64 restatements ----
# The golden fixtures are the numpy restatement in FP64 and the oracle's FP64 instantiation
# follows the reference built with DP=1, so the bound is FP64 round-off: copies, permutations
# and macrovars bit for bit, the closed-form collision within 1e-13 (the eddy viscosity, a
# small difference of squares, within 1e-10).

def g64(golden, name):
    return np.ascontiguousarray(golden[name].astype(np.float64))


def test_f64_fequil3_postcoll(golden, nl):
    p = "q%d_" % nl
    s = (slice(1, -1),) * 3
    for ibgk, key in ((3, "fequil3"), (2, "fequil2")):
        L = mk(nl, ibgk=ibgk)
        feq = L.empty_f(torch.float64)
        L.fequil3(feq, *(dev(g64(golden, p + n)) for n in ("rho", "u", "v", "w")))
        assert rel_l2(host(feq)[s], golden[p + key][s]) < 1e-14
    for ihrr in (0, 1):
        for ivr in (0, 1):
            L = mk(nl, ihrr=ihrr, ivreman=ivr)
            f = dev(g64(golden, p + "f"))
            tau = dev(np.full((NZ + 2, NY + 2, NX + 2), 3 * 1e-4 + 0.5))
            L.postcoll(f, tau, *(dev(g64(golden, p + n)) for n in ("rho", "u", "v", "w")))
            fo, to = host(f), host(tau)
            assert rel_l2(fo[s], golden[p + "postcoll_h%d_v%d_f" % (ihrr, ivr)][s]) < 1e-13
            assert rel_l2(to[s] - 0.5, golden[p + "postcoll_h%d_v%d_tau" % (ihrr, ivr)][s] - 0.5) < 1e-10
            np.testing.assert_array_equal(fo[0], g64(golden, p + "f")[0])


def test_f64_params_reach_the_kernels(golden, nl):
    """kinevisc converted from the FP32 lbm_params differs from the double one; the
    FP64 relaxation time shows the difference (3 x 2.5e-12) until set_params_f64."""
    p = "q%d_" % nl
    s = (slice(1, -1),) * 3
    L = mk(nl)
    taus = []
    for nu in (float(np.float32(1e-4)), 1e-4):
        L.set_params_f64(kinevisc=nu)
        tau = dev(np.zeros((NZ + 2, NY + 2, NX + 2)))
        L.vreman(dev(g64(golden, p + "vreman_in")), tau)
        taus.append(host(tau)[s])
    d = np.abs(taus[0] - taus[1])
    assert np.allclose(d, 3 * (1e-4 - float(np.float32(1e-4))), rtol=1e-3, atol=0)
    assert rel_l2(taus[1] - 0.5, golden[p + "vreman_tau"][s] - 0.5) < 1e-10


def test_f64_drift_macrovars_bitexact(golden, nl):
    p = "q%d_" % nl
    L = mk(nl)
    o = O.Oracle(ocfg(nl), np.float64)
    fin = g64(golden, p + "f")
    fout = L.empty_f(torch.float64)
    L.drift(fout, dev(fin))
    ref = o.zeros_f()
    o.drift(ref, fin)
    np.testing.assert_array_equal(host(fout), ref)
    out = [L.empty_s(torch.float64) for _ in range(4)]
    L.macrovars(*out, dev(fin))
    refm = [o.zeros_s() for _ in range(4)]
    o.macrovars(*refm, fin)
    for a, b in zip(out, refm):
        np.testing.assert_array_equal(host(a), b)


def test_f64_regularization_vreman_fneq_f(golden, nl):
    p = "q%d_" % nl
    s = (slice(1, -1),) * 3
    L = mk(nl)
    f = dev(g64(golden, p + "f"))
    L.regularization(f, dev(g64(golden, p + "fequil3")), *(dev(g64(golden, p + n)) for n in ("u", "v", "w")))
    assert rel_l2(host(f)[s], golden[p + "regularization"][s]) < 1e-13
    tau = L.empty_s(torch.float64)
    L.vreman(dev(g64(golden, p + "vreman_in")), tau)
    assert rel_l2(host(tau)[s] - 0.5, golden[p + "vreman_tau"][s] - 0.5) < 1e-10
    a, b = g64(golden, p + "f"), g64(golden, p + "fequil3")
    f = dev(a)
    L.compute_fneq(f, dev(b))
    np.testing.assert_array_equal(host(f), a - b)
    L.compute_f(f, dev(b))
    np.testing.assert_array_equal(host(f), b + (a - b))


@pytest.mark.parametrize("codes", [(1, 0, 12), (0, 0, 0), (11, 22, 12), (22, 21, 11), (12, 11, 22), (1, 11, 22)])
def test_f64_boundarycond(golden, nl, codes):
    p = "q%d_" % nl
    ib, jb, kb = codes
    udir = 10.0 if ib == 1 else 0.0
    L = mk(nl, ibnd=ib, jbnd=jb, kbnd=kb, udir=udir)
    f1, f2 = g64(golden, p + "bc_f1"), g64(golden, p + "bc_f2")
    uvel = g64(golden, p + "bc_uvel")
    d1, d2 = dev(f1), dev(f2)
    L.boundarycond(d1, d2, dev(uvel))
    o = O.Oracle(ocfg(nl, ibnd=ib, jbnd=jb, kbnd=kb, udir=udir), np.float64)
    r1, r2 = f1.copy(), f2.copy()
    o.boundarycond(r1, r2, uvel)
    out = host(d1)
    if ib == 1:
        # the inflow ghosts hold cos/sin of udir, evaluated on the device and on the host
        np.testing.assert_array_equal(out[:, :, 1:], r1[:, :, 1:])
        assert rel_l2(out, r1) < 1e-15
    else:
        np.testing.assert_array_equal(out, r1)
    np.testing.assert_array_equal(host(d2), f2)


def test_f64_solids_fillghosts_turbulence(golden, nl):
    p = "q%d_" % nl
    L = mk(nl)
    f = dev(g64(golden, p + "f"))
    L.solids(f, dev(golden[p + "solids_mask"].astype(np.int32)))
    np.testing.assert_array_equal(host(f), golden[p + "solids"])
    f = dev(g64(golden, p + "f"))
    L.fillghosts(f)
    np.testing.assert_array_equal(host(f), golden[p + "fillghosts"])
    df = torch.zeros((NZ, NY, nl), dtype=torch.float64, device="cuda")
    uu, vv, ww = (dev(g64(golden, p + n)) for n in ("turb_uu", "turb_vv", "turb_ww"))
    L.inflow_turbulence_forcing(df, *(dev(g64(golden, p + n)) for n in ("rho", "u", "v", "w")), uu, vv, ww,
                                1e-2, 7, 4)
    out = host(df)
    assert rel_l2(out, golden[p + "turb_df_it7"]) < 1e-12
    f = dev(g64(golden, p + "f"))
    L.inflow_turbulence_apply(f, df)
    o = O.Oracle(ocfg(nl), np.float64)
    ref = g64(golden, p + "f")
    o.turbulence_apply(ref, out)
    np.testing.assert_array_equal(host(f), ref)


def test_f64_forcings_apply(nl):
    from lbm_b200 import Lbm, Params
    cfg = O.Config(13, 7, 6, nl)
    rng = np.random.default_rng(5)
    f = rng.uniform(0.0, 0.1, cfg.fshape)
    rho = 1.0 + 0.01 * rng.standard_normal(cfg.sshape)
    u, v, w = (0.03 * rng.standard_normal(cfg.sshape) for _ in range(3))
    F = 1e-4 * rng.standard_normal(cfg.sshape + (3,))
    ref = f.copy()
    O.Oracle(cfg, np.float64).forcings_apply(ref, F, rho, u, v, w)
    L = Lbm(Params(nx=13, ny=7, nz=6, nl=nl, iturb_pos=3))
    fg = dev(f)
    L.forcings_apply(fg, dev(F), *(dev(a) for a in (rho, u, v, w)))
    # the oracle forms feq1 - feq0 as a difference of two O(0.05) values
    assert np.abs(host(fg) - ref).max() < 1e-15


def test_f64_mixed_precision_refused(nl):
    from lbm_b200 import LbmError
    L = mk(nl)
    with pytest.raises(LbmError):
        L.drift(L.empty_f(torch.float64), L.empty_f())                     # float64 f, float32 feq
    with pytest.raises(LbmError):
        L.macrovars(*(L.empty_s() for _ in range(4)), L.empty_f(torch.float64))
