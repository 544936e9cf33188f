"""Pin the C++ oracle against the independent numpy restatement's fixtures.

The fixtures (tests/golden/golden_small.npz, made by make_golden.py) come
from a second, vectorised restatement of the reference routines.  The FP64
oracle must agree to round-off; the FP32 oracle to single-precision level,
and exactly where the routine only moves values (drift, boundary copies,
solids, fillghosts)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import rel_l2

NX, NY, NZ = 4, 3, 3


def cfg(nl, **kw):
    base = dict(nx=NX, ny=NY, nz=NZ, nl=nl, iturb_pos=3, nrturb=4, ampl=1e-2)
    base.update(kw)
    return O.Config(**base)


def arr(g, name, dt):
    return np.ascontiguousarray(g[name].astype(dt))


TOL = {np.float64: 1e-12, np.float32: 2e-6}


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("nl", [19, 27])
class TestSingleCall:
    def test_fequil3(self, golden, nl, dt):
        p = "q%d_" % nl
        for ibgk, key in ((3, "fequil3"), (2, "fequil2")):
            o = O.Oracle(cfg(nl, ibgk=ibgk), dt)
            feq = o.zeros_f()
            o.fequil3(feq, *(arr(golden, p + n, dt) for n in ("rho", "u", "v", "w")))
            assert rel_l2(feq[1:-1, 1:-1, 1:-1], golden[p + key][1:-1, 1:-1, 1:-1]) < TOL[dt]

    @pytest.mark.parametrize("ihrr", [0, 1])
    @pytest.mark.parametrize("ivr", [0, 1])
    def test_postcoll(self, golden, nl, dt, ihrr, ivr):
        p = "q%d_" % nl
        o = O.Oracle(cfg(nl, ihrr=ihrr, ivreman=ivr), dt)
        f = arr(golden, p + "f", dt)
        tau = np.full(o.cfg.sshape, 3 * 1e-4 + 0.5, dt)
        o.postcoll(f, tau, *(arr(golden, p + n, dt) for n in ("rho", "u", "v", "w")))
        ref_f = golden[p + "postcoll_h%d_v%d_f" % (ihrr, ivr)]
        ref_t = golden[p + "postcoll_h%d_v%d_tau" % (ihrr, ivr)]
        assert rel_l2(f[1:-1, 1:-1, 1:-1], ref_f[1:-1, 1:-1, 1:-1]) < TOL[dt]
        assert rel_l2(tau[1:-1, 1:-1, 1:-1] - 0.5, ref_t[1:-1, 1:-1, 1:-1] - 0.5) < 50 * TOL[dt]

    def test_drift_exact(self, golden, nl, dt):
        p = "q%d_" % nl
        o = O.Oracle(cfg(nl), dt)
        fd = o.zeros_f()
        o.drift(fd, arr(golden, p + "f", dt))
        np.testing.assert_array_equal(fd, golden[p + "drift"].astype(dt))

    def test_macrovars(self, golden, nl, dt):
        p = "q%d_" % nl
        o = O.Oracle(cfg(nl), dt)
        out = [o.zeros_s() for _ in range(4)]
        o.macrovars(*out, arr(golden, p + "f", dt))
        for a, b in zip(out, golden[p + "macro"]):
            assert rel_l2(a, b) < TOL[dt]

    def test_regularization(self, golden, nl, dt):
        p = "q%d_" % nl
        o = O.Oracle(cfg(nl), dt)
        f = arr(golden, p + "f", dt)
        feq = arr(golden, p + "fequil3", dt)
        o.regularization(f, feq, *(arr(golden, p + n, dt) for n in ("u", "v", "w")))
        ref = golden[p + "regularization"]
        assert rel_l2(f[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1]) < 20 * TOL[dt]

    def test_vreman(self, golden, nl, dt):
        p = "q%d_" % nl
        o = O.Oracle(cfg(nl), dt)
        tau = o.zeros_s()
        o.vreman(arr(golden, p + "vreman_in", dt), tau)
        ref = golden[p + "vreman_tau"]
        assert rel_l2(tau[1:-1, 1:-1, 1:-1] - 0.5, ref[1:-1, 1:-1, 1:-1] - 0.5) < 50 * TOL[dt]

    @pytest.mark.parametrize("codes", [(1, 0, 12), (0, 0, 0), (11, 22, 12), (22, 21, 11), (12, 11, 22), (1, 11, 22)])
    def test_boundarycond(self, golden, nl, dt, codes):
        p = "q%d_" % nl
        ib, jb, kb = codes
        o = O.Oracle(cfg(nl, ibnd=ib, jbnd=jb, kbnd=kb, udir=10.0 if ib == 1 else 0.0), dt)
        f1 = arr(golden, p + "bc_f1", dt)
        f2 = arr(golden, p + "bc_f2", dt)
        o.boundarycond(f1, f2, arr(golden, p + "bc_uvel", dt))
        ref = golden[p + "bc_%d_%d_%d" % codes]
        if ib == 1:
            # inflow ghost plane involves arithmetic; the rest is pure copies
            assert rel_l2(f1, ref) < TOL[dt]
            np.testing.assert_array_equal(f1[:, :, 1:], ref[:, :, 1:].astype(dt))
        else:
            np.testing.assert_array_equal(f1, ref.astype(dt))
        np.testing.assert_array_equal(f2, golden[p + "bc_f2"].astype(dt))

    def test_solids_and_fillghosts(self, golden, nl, dt):
        p = "q%d_" % nl
        o = O.Oracle(cfg(nl), dt)
        f = arr(golden, p + "f", dt)
        o.solids(f, np.ascontiguousarray(golden[p + "solids_mask"]))
        np.testing.assert_array_equal(f, golden[p + "solids"].astype(dt))
        f = arr(golden, p + "f", dt)
        o.fillghosts(f)
        np.testing.assert_array_equal(f, golden[p + "fillghosts"].astype(dt))

    def test_turbulence_forcing(self, golden, nl, dt):
        p = "q%d_" % nl
        o = O.Oracle(cfg(nl), dt)
        df = np.zeros((NZ, NY, nl), dt)
        o.turbulence_forcing(df, *(arr(golden, p + n, dt) for n in ("rho", "u", "v", "w")),
                             *(arr(golden, p + n, dt) for n in ("turb_uu", "turb_vv", "turb_ww")), 7)
        ref = golden[p + "turb_df_it7"]
        # df is a difference of two O(w) equilibria: FP32 keeps ~1e-7*w absolute
        tol = 1e-12 if dt == np.float64 else 2e-3
        assert rel_l2(df, ref) < tol


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("nl", [19, 27])
def test_init_and_run(golden, nl, dt):
    p = "q%d_" % nl
    c = cfg(nl, nx=6, ny=4, nz=4, lsolids=True, lturb=True)
    o = O.Oracle(c, dt)
    rho, u, v, w = (np.ascontiguousarray(a.astype(dt)) for a in golden[p + "run_in"])
    uvel = arr(golden, p + "run_uvel", dt)
    fA, fB = o.zeros_f(), o.zeros_f()
    o.init(fA, fB, rho, u, v, w, uvel)
    tol = TOL[dt]
    assert rel_l2(fA, golden[p + "run_init_fA"]) < tol
    assert rel_l2(fB, golden[p + "run_init_fB"]) < tol
    tau = np.full(c.sshape, 3 * 1e-4 + 0.5, dt)
    uu, vv, ww = (np.ascontiguousarray(a.astype(dt)) for a in golden[p + "run_turb"])
    o.run(fA, fB, rho, u, v, w, tau, uvel, 6, blanking=np.ascontiguousarray(golden[p + "run_mask"]),
          uu=uu, vv=vv, ww=ww)
    tol = 1e-11 if dt == np.float64 else 5e-6
    assert rel_l2(fA, golden[p + "run_f1"]) < tol
    assert rel_l2(fB, golden[p + "run_f2"]) < tol
    assert rel_l2(rho, golden[p + "run_rho"]) < tol
    vel = np.stack([u, v, w])[:, 1:-1, 1:-1, 1:-1]
    ref = np.stack([golden[p + "run_" + n] for n in "uvw"])[:, 1:-1, 1:-1, 1:-1]
    assert rel_l2(vel, ref) < 20 * tol
