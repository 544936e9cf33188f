"""Adjoint kernels and the checkpointed reverse sweep.

Each adjoint kernel passes a dot-product test, <y^, J x> = <J^T y^, x>, with
J x from central differences of the FP64 oracle's forward kernel.  The full
sweep's gradient of a probe-misfit loss matches central differences of the
FP64 oracle's time loop along 8 seeded directions (4 in the initial f, 4 in
the inflow profile) to a relative 1e-4; at the adjoint workload's full size
the central differences come from the FP64 forward run on the GPU."""
import numpy as np
import pytest

from lbm_b200 import workloads as W
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.float64)


def near_equilibrium(o, rng, amp=0.02, noise=2e-3):
    """a state f with rho ~ 1 and |u| ~ 0.05, plus non-equilibrium noise"""
    cfg = o.cfg
    rho = 1.0 + amp * rng.standard_normal(cfg.sshape)
    u = 0.05 + amp * rng.standard_normal(cfg.sshape)
    v = amp * rng.standard_normal(cfg.sshape)
    w = amp * rng.standard_normal(cfg.sshape)
    feq = o.zeros_f()
    o.fequil3(feq, rho, u, v, w)
    t = O.tables(cfg.nl, np.float64)
    inner = (slice(1, -1),) * 3
    f = np.broadcast_to(t["w"], cfg.fshape).copy()
    f[inner] = feq[inner]
    f += noise * rng.standard_normal(cfg.fshape) * t["w"]
    return f, rho, u, v, w


def config(nl, **kw):
    base = dict(ibnd=1, jbnd=0, kbnd=12, iturb_pos=2)
    base.update(kw)
    return O.Config(9, 7, 6, nl, **base)


def lbm_of(cfg):
    from lbm_b200 import Lbm, Params
    return Lbm(Params(nx=cfg.nx, ny=cfg.ny, nz=cfg.nz, nl=cfg.nl, ibnd=cfg.ibnd, jbnd=cfg.jbnd, kbnd=cfg.kbnd,
                      iturb_pos=cfg.iturb_pos, ivreman=cfg.ivreman, kinevisc=cfg.kinevisc))


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("nl", [19, 27])
@pytest.mark.parametrize("ivreman", [1, 0])
def test_postcoll_adjoint_dot_product(nl, ivreman):
    cfg = config(nl, ivreman=ivreman)
    o = O.Oracle(cfg, np.float64)
    rng = np.random.default_rng(7 + nl + ivreman)
    f, rho, u, v, w = near_equilibrium(o, rng)
    tau = np.full(cfg.sshape, 3e-4 + 0.5 if ivreman else 0.56)
    x = [rng.standard_normal(a.shape) * s for a, s in ((f, 1e-3), (rho, 1e-3), (u, 1e-3), (v, 1e-3), (w, 1e-3))]
    yh = rng.standard_normal(cfg.fshape)

    def fwd(sgn, eps=1e-4):
        ff = f + sgn * eps * x[0]
        args = [a + sgn * eps * d for a, d in zip((rho, u, v, w), x[1:])]
        o.postcoll(ff, tau.copy(), *args)
        return ff
    jx = (fwd(+1) - fwd(-1)) / 2e-4
    lhs = float((yh * jx).sum())
    L = lbm_of(cfg)
    fh = cuda(yh)
    R = [cuda(a) for a in (rho, u, v, w)]
    Rh = [L.empty_s() for _ in range(4)]
    L.postcoll_adj(fh, cuda(f), *R, *Rh, tau=cuda(tau))
    rhs = float((host(fh) * x[0]).sum()) + sum(float((host(a) * d).sum()) for a, d in zip(Rh, x[1:]))
    assert rel(lhs, rhs) < 1e-4, (lhs, rhs)


@pytest.mark.parametrize("nl", [19, 27])
def test_macrovars_adjoint_dot_product(nl):
    cfg = config(nl)
    o = O.Oracle(cfg, np.float64)
    rng = np.random.default_rng(3)
    f = near_equilibrium(o, rng)[0]
    x = rng.standard_normal(cfg.fshape) * 1e-3
    yh = [rng.standard_normal(cfg.sshape) for _ in range(4)]

    def fwd(sgn, eps=1e-4):
        R = [np.zeros(cfg.sshape) for _ in range(4)]
        o.macrovars(*R, f + sgn * eps * x)
        return R
    p, m = fwd(+1), fwd(-1)
    lhs = sum(float((a * (b - c)).sum()) for a, b, c in zip(yh, p, m)) / 2e-4
    L = lbm_of(cfg)
    fh = L.empty_f()
    L.macrovars_adj(fh, *[cuda(a) for a in yh], cuda(f))
    rhs = float((host(fh) * x).sum())
    assert rel(lhs, rhs) < 1e-4, (lhs, rhs)


@pytest.mark.parametrize("nl", [19, 27])
def test_drift_adjoint_is_the_transpose(nl):
    cfg = config(nl)
    o = O.Oracle(cfg, np.float64)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(cfg.fshape)
    yh = rng.standard_normal(cfg.fshape)
    out = rng.standard_normal(cfg.fshape)           # drift keeps the ghost cells of its output
    o.drift(out, x)
    base = np.zeros(cfg.fshape)
    o.drift(base, np.zeros(cfg.fshape))
    lhs = float((yh * out).sum())
    L = lbm_of(cfg)
    fin, fout = L.empty_f(), cuda(yh)
    L.drift_adj(fin, fout)
    inner = (slice(1, -1),) * 3
    ghosts_out = out.copy()
    ghosts_out[inner] = 0.0
    # <yh, drift(x) + kept ghosts> = <drift^T yh, x> + <yh on ghosts, old ghosts>
    rhs = float((host(fin) * x).sum()) + float((yh * ghosts_out).sum())
    assert rel(lhs, rhs) < 1e-6, (lhs, rhs)
    assert np.all(host(fout)[inner] == 0.0)


@pytest.mark.parametrize("codes", [(1, 0, 12), (1, 0, 21), (0, 0, 0), (11, 22, 12), (1, 11, 22), (0, 12, 0)])
@pytest.mark.parametrize("nl", [19, 27])
def test_boundarycond_adjoint_dot_product(codes, nl):
    ib, jb, kb = codes
    cfg = config(nl, ibnd=ib, jbnd=jb, kbnd=kb)
    o = O.Oracle(cfg, np.float64)
    rng = np.random.default_rng(11)
    f1, f2 = rng.standard_normal(cfg.fshape), rng.standard_normal(cfg.fshape)
    uvel = 0.05 + 0.01 * rng.standard_normal(cfg.nz)
    x1, x2 = rng.standard_normal(cfg.fshape), rng.standard_normal(cfg.fshape)
    xu = rng.standard_normal(cfg.nz)
    yh = rng.standard_normal(cfg.fshape)

    def bc(a1, a2, uv):
        a1 = a1.copy()
        o.boundarycond(a1, a2.copy(), uv)
        return a1
    jx = bc(f1 + x1, f2 + x2, uvel + xu) - bc(f1, f2, uvel)     # affine map: exact difference
    lhs = float((yh * jx).sum())
    L = lbm_of(cfg)
    f1h, f2h = cuda(yh), L.empty_f()
    uh = torch.zeros(cfg.nz, device="cuda")
    L.boundarycond_adj(f1h, f2h, uh)
    rhs = float((host(f1h) * x1).sum() + (host(f2h) * x2).sum() + (host(uh) * xu).sum())
    assert rel(lhs, rhs) < 1e-5, (lhs, rhs)


# ---- the whole reverse sweep -------------------------------------------------------------
CASE = W.Workload("adjoint_small", 20, 10, 8, 19, steps=12, sphere=(9, 5, 4, 2), noise=1e-3)


def problem(wl, checkpoint):
    from lbm_b200 import Params
    from lbm_b200.adjoint import ProbeProblem, initial_state
    p = Params(nx=wl.nx, ny=wl.ny, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=2,
               kinevisc=wl.kinevisc)
    blank = torch.from_numpy(W.blanking(wl)).cuda()
    pb = ProbeProblem(p, W.probe_cells(wl, 24, 1), wl.steps, blanking=blank, checkpoint=checkpoint)
    rho, u, v, w = (cuda(a) for a in W.initial_macro(wl))
    uvel = cuda(W.inflow_profile(wl))
    f1, f2 = initial_state(pb.lbm, rho, u, v, w, uvel)
    # spin up away from the exact equilibrium of the initial state, where the
    # Vreman viscosity (homogeneous of degree one in the non-equilibrium moments)
    # has no derivative
    R = pb._macro(f1)
    for _ in range(30):
        f1, f2 = pb._step(f1, f2, R, uvel)
    return pb, f1, f2, uvel


def oracle_probe_u(wl, probes, f1, f2, uvel):
    cfg = O.Config(wl.nx, wl.ny, wl.nz, wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=2, lsolids=True,
                   kinevisc=wl.kinevisc)
    o = O.Oracle(cfg, np.float64)
    fA, fB = f1.copy(), f2.copy()
    R = [np.zeros(cfg.sshape) for _ in range(4)]
    o.macrovars(*R, fA)
    tau = np.full(cfg.sshape, 3 * wl.kinevisc + 0.5)
    o.run(fA, fB, *R, tau, uvel, wl.steps, blanking=W.blanking(wl))
    i, j, k = probes[:, 0], probes[:, 1], probes[:, 2]
    return np.stack([R[q][k, j, i] for q in (1, 2, 3)], axis=1)


def oracle_loss(wl, probes, f1, f2, uvel, target):
    return float(((oracle_probe_u(wl, probes, f1, f2, uvel) - target) ** 2).sum())


@pytest.mark.parametrize("checkpoint", [5, 12])
def test_gradient_matches_fp64_finite_differences(checkpoint):
    wl = CASE
    pb, f1, f2, uvel = problem(wl, checkpoint)
    # target: the same run with the inflow profile perturbed by smooth seeded noise (5e-3)
    truth = pb.forward(f1, f2, uvel + cuda(W.inflow_perturbation(wl.nz, 2, 5e-3)), keep=False)
    pb.forward(f1, f2, uvel)
    F1, F2, U, T = host(f1), host(f2), host(uvel), host(truth)
    # the sweep is seeded with the FP64 run's misfit, so the test measures the
    # adjoint itself rather than the FP32 rounding of the small misfits
    u64 = oracle_probe_u(wl, pb.probes, F1, F2, U)
    gf, gu = pb.backward(cuda(2.0 * (u64 - T)))
    gf, gu = host(gf), host(gu)
    rng = np.random.default_rng(42)
    inner = (slice(1, -1),) * 3
    worst = 0.0
    for d in range(8):
        df, du = np.zeros_like(F1), np.zeros_like(U)
        if d < 4:
            df[inner] = 1e-6 * rng.standard_normal(df[inner].shape)
        else:
            du = 1e-6 * rng.standard_normal(U.shape)
        fd = (oracle_loss(wl, pb.probes, F1 + df, F2, U + du, T)
              - oracle_loss(wl, pb.probes, F1 - df, F2, U - du, T)) / 2.0
        ad = float((gf * df).sum() + (gu * du).sum())
        worst = max(worst, rel(fd, ad))
        assert rel(fd, ad) < 1e-4, (d, fd, ad)
    print("worst relative error of 8 directional derivatives:", worst)
    pb.close()


def test_autograd_function_gives_the_sweep_gradient():
    from tests.adjoint_harness import probe_loss
    wl = CASE.with_(steps=6)
    pb, f1, f2, uvel = problem(wl, 4)
    target = pb.forward(f1, f2, uvel + cuda(W.inflow_perturbation(wl.nz, 3, 5e-3)), keep=False)
    x1 = f1.clone().requires_grad_(True)
    xu = uvel.clone().requires_grad_(True)
    loss = probe_loss(x1, xu, f2, pb, target)
    g1, gu = torch.autograd.grad(loss, (x1, xu))
    u = pb.forward(f1, f2, uvel)
    r1, ru = pb.backward(2.0 * (u - target))
    assert torch.equal(g1, r1) and torch.equal(gu, ru)
    assert float(loss.detach()) > 0 and float(gu.abs().sum()) > 0
    pb.close()


def test_autograd_function_with_the_state_layout_sweep():
    """The same torch.autograd wrapper around the fused-forward problem: its
    gradient is the state-layout sweep's (f1 bit for bit)."""
    from tests.adjoint_harness import probe_loss
    wl = CASE.with_(steps=6)
    pb, f1, f2, uvel = problem(wl, 4)
    target = pb.forward(f1, f2, uvel + cuda(W.inflow_perturbation(wl.nz, 3, 5e-3)), keep=False)
    pb.close()
    fb = fused_problem(wl, 4, None)
    x1 = f1.clone().requires_grad_(True)
    xu = uvel.clone().requires_grad_(True)
    loss = probe_loss(x1, xu, f2, fb, target)
    g1, gu = torch.autograd.grad(loss, (x1, xu))
    u = fb.forward(f1, f2, uvel)
    r1, ru = fb.backward((2.0 * (u.double() - target.double())).float())
    assert torch.equal(g1, r1)
    # uvelhat is summed with atomics, whose order may differ between two sweeps
    assert float((gu - ru).abs().max()) <= 1e-6 * float(ru.abs().max()) + 1e-12
    assert float(loss.detach()) > 0 and float(g1.abs().sum()) > 0
    fb.close()


def test_fused_adjoints_equal_the_chained_ones():
    """macrovars_drift_adj == macrovars_adj then drift_adj (macrovars adjoints at
    interior cells); postcoll_adj with blanking == solids then postcoll_adj."""
    cfg = config(19)
    o = O.Oracle(cfg, np.float64)
    rng = np.random.default_rng(9)
    f, rho, u, v, w = near_equilibrium(o, rng)
    L = lbm_of(cfg)
    F = cuda(f)
    R = [L.empty_s() for _ in range(4)]
    L.macrovars(*R, F)
    inner = (slice(1, -1),) * 3
    Rh = []
    for _ in range(4):
        a = np.zeros(cfg.sshape)
        a[inner] = rng.standard_normal(a[inner].shape)
        Rh.append(cuda(a))
    y = rng.standard_normal(cfg.fshape)
    a_in, a_out = cuda(y * 0.5), cuda(y)
    b_in, b_out = a_in.clone(), a_out.clone()
    L.macrovars_adj(a_out, *Rh, F)
    L.drift_adj(a_in, a_out)
    L.macrovars_drift_adj(b_in, b_out, *Rh, *R)
    np.testing.assert_allclose(host(b_in), host(a_in), rtol=1e-5, atol=1e-6)
    assert torch.equal(a_out, b_out)
    blank = torch.from_numpy((rng.uniform(size=cfg.sshape) < 0.3).astype(np.int32)).cuda()
    Rf = [cuda(a) for a in (rho, u, v, w)]
    g1, g2 = cuda(y), cuda(y)
    h1, h2 = [L.empty_s() for _ in range(4)], [L.empty_s() for _ in range(4)]
    L.solids(g1, blank)
    L.postcoll_adj(g1, F, *Rf, *h1)
    L.postcoll_adj(g2, F, *Rf, *h2, blanking=blank)
    assert torch.equal(g1, g2) and all(torch.equal(p, q) for p, q in zip(h1, h2))


# ---- the reverse sweep in the state layout (forward by the fused step) -----------------
def fused_problem(wl, checkpoint, spin_from):
    from lbm_b200 import Params
    from lbm_b200.adjoint import FusedProbeProblem
    p = Params(nx=wl.nx, ny=wl.ny, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=2,
               kinevisc=wl.kinevisc)
    blank = torch.from_numpy(W.blanking(wl)).cuda()
    return FusedProbeProblem(p, W.probe_cells(wl, 24, 1), wl.steps, blanking=blank, checkpoint=checkpoint)


@pytest.mark.parametrize("nl", [19, 27])
def test_state_layout_sweep_matches_fp64_finite_differences(nl):
    wl = CASE.with_(nl=nl)
    pb, f1, f2, uvel = problem(wl, 5)           # spun-up initial state (per-call path)
    fb = fused_problem(wl, 5, None)
    truth = fb.forward(f1, f2, uvel + cuda(W.inflow_perturbation(wl.nz, 2, 5e-3)), keep=False)
    fb.forward(f1, f2, uvel)
    F1, F2, U, T = host(f1), host(f2), host(uvel), host(truth)
    u64 = oracle_probe_u(wl, fb.probes, F1, F2, U)
    gf, gu = fb.backward(cuda(2.0 * (u64 - T)))
    gf, gu = host(gf), host(gu)
    # the per-call sweep gives the same gradient
    pb.forward(f1, f2, uvel)
    rf, ru = (host(t) for t in pb.backward(cuda(2.0 * (u64 - T))))
    assert np.abs(gf - rf).max() <= 1e-4 * np.abs(rf).max() and np.abs(gu - ru).max() <= 1e-4 * np.abs(ru).max()
    rng = np.random.default_rng(43)
    inner = (slice(1, -1),) * 3
    for d in range(8):
        df, du = np.zeros_like(F1), np.zeros_like(U)
        if d < 4:
            df[inner] = 1e-6 * rng.standard_normal(df[inner].shape)
        else:
            du = 1e-6 * rng.standard_normal(U.shape)
        fd = (oracle_loss(wl, fb.probes, F1 + df, F2, U + du, T) - oracle_loss(wl, fb.probes, F1 - df, F2, U - du, T)) / 2
        ad = float((gf * df).sum() + (gu * du).sum())
        assert rel(fd, ad) < 1e-4, (d, fd, ad)
    pb.close()
    fb.close()


@pytest.mark.parametrize("codes", [(11, 22, 12), (0, 0, 0), (1, 11, 22), (0, 12, 0), (11, 0, 22), (1, 0, 0),
                                   (1, 0, 21), (1, 0, 12)])
@pytest.mark.parametrize("nl", [19, 27])
def test_state_layout_sweep_matches_per_call_sweep_for_boundary_codes(codes, nl):
    """Closed faces, edges and corners, periodic axes and inflow: the boundary
    adjoint reaches the cells next to every face.  With periodic j the state
    adjoint reads ghost rows as rows ny and 1 (no j copies); closed i and k with
    periodic j make edges along j; inflow i, periodic j and closed k take the
    folded boundary adjoint."""
    ib, jb, kb = codes
    wl = CASE.with_(nl=nl, ibnd=ib, jbnd=jb, kbnd=kb, steps=8)
    pb, f1, f2, uvel = problem(wl, 3)
    fb = fused_problem(wl, 3, None)
    rng = np.random.default_rng(7)
    uhat = cuda(rng.standard_normal((len(fb.probes), 3)))
    fb.forward(f1, f2, uvel)
    gf, gu = (host(t) for t in fb.backward(uhat))
    pb.forward(f1, f2, uvel)
    rf, ru = (host(t) for t in pb.backward(uhat))
    assert np.abs(rf).max() > 0
    assert np.abs(gf - rf).max() <= 1e-4 * np.abs(rf).max(), codes
    if ib == 1:
        assert np.abs(gu - ru).max() <= 1e-4 * np.abs(ru).max()
    pb.close()
    fb.close()


def test_state_layout_sweep_refuses_unsupported_states():
    from lbm_b200 import LbmError, Params
    from lbm_b200.adjoint import FusedProbeProblem
    with pytest.raises(ValueError):
        FusedProbeProblem(Params(nx=8, ny=6, nz=6, nl=19, iturb_pos=2, storage="f16"), [(1, 1, 1)], 2)
    from lbm_b200 import Lbm
    L = Lbm(Params(nx=8, ny=6, nz=6, nl=19, iturb_pos=2, ihrr=0))
    a, b = L.empty_state(), L.empty_state()
    with pytest.raises(LbmError, match="ihrr"):
        L.state_adjoint_step(a, b, a.clone(), True, torch.zeros(6, device="cuda"))


def test_full_size_gradient_matches_fp64_gpu_finite_differences():
    """The adjoint workload at its own size: D3Q19 256x128x128, sphere r = 16,
    200 probes, 100 steps, checkpoints every 10.  The state-layout sweep's
    gradient (FP32 fused forward) against central differences of the FP64
    forward run on the GPU through the _f64 entry points (the reference's DP
    build), along 8 seeded directions (4 in f1, 4 in uvel), each within 1e-4."""
    from lbm_b200 import Params
    from lbm_b200.adjoint import FusedProbeProblem, ProbeProblem, initial_state
    wl = W.ADJOINT_Q19
    p = Params(nx=wl.nx, ny=wl.ny, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=10,
               kinevisc=wl.kinevisc)
    blank = torch.from_numpy(W.blanking(wl)).cuda()
    probes = W.probe_cells(wl, 200, 0)
    spin = ProbeProblem(p, probes, wl.steps, blanking=blank, checkpoint=10)
    rho, u, v, w = (torch.from_numpy(x).cuda() for x in W.initial_macro(wl))
    uvel = torch.from_numpy(W.inflow_profile(wl)).cuda()
    f1, f2 = initial_state(spin.lbm, rho, u, v, w, uvel)
    R = spin._macro(f1)
    for _ in range(20):                       # leave the exact initial equilibrium
        f1, f2 = spin._step(f1, f2, R, uvel)
    spin.close()
    p64 = ProbeProblem(p, probes, wl.steps, blanking=blank, dtype=torch.float64)
    F1, F2, U = f1.double(), f2.double(), uvel.double()
    dU = torch.from_numpy(W.inflow_perturbation(wl.nz, 0, 5e-3)).cuda().double()
    T = p64.forward(F1, F2, U + dU, keep=False)
    u64 = p64.forward(F1, F2, U, keep=False)
    fb = FusedProbeProblem(p, probes, wl.steps, blanking=blank, checkpoint=10)
    fb.forward(f1, f2, uvel)
    gf, gu = (t.double() for t in fb.backward((2.0 * (u64 - T)).float()))
    fb.close()

    def loss(a, b):
        return float(((p64.forward(a, F2, b, keep=False) - T) ** 2).sum())

    gen = torch.Generator(device="cuda").manual_seed(44)
    inner = (slice(1, -1),) * 3
    worst = 0.0
    for d in range(8):
        df, du = torch.zeros_like(F1), torch.zeros_like(U)
        if d < 4:
            df[inner] = 1e-6 * torch.randn(df[inner].shape, generator=gen, device="cuda", dtype=torch.float64)
        else:
            du = 1e-6 * torch.randn(U.shape, generator=gen, device="cuda", dtype=torch.float64)
        fd = (loss(F1 + df, U + du) - loss(F1 - df, U - du)) / 2.0
        ad = float((gf * df).sum() + (gu * du).sum())
        worst = max(worst, rel(fd, ad))
        assert rel(fd, ad) < 1e-4, (d, fd, ad)
    print("worst relative error of 8 directional derivatives at 256x128x128:", worst)
    p64.close()
