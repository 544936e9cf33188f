"""Analytic known answers that pin the oracle independently of any restatement.

Identities of the D3Q19/D3Q27 lattices and of the reference step
(mod_D3Q27setup.F90, m_fequil3_kernel.F90, m_postcoll_kernel.F90,
m_drift_kernel.F90, m_solids.F90): weight moments, equilibrium moments,
fixed points, conservation, permutation and involution properties."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("nl", [19, 27])
def test_lattice_moments(nl):
    t = O.tables(nl, np.float64)
    w, c = t["w"], np.stack([t["cx"], t["cy"], t["cz"]], 1).astype(np.float64)
    assert abs(w.sum() - 1.0) < 1e-15
    np.testing.assert_allclose(w @ c, 0.0, atol=1e-16)
    np.testing.assert_allclose(np.einsum("l,lp,lq->pq", w, c, c), np.eye(3) / 3.0, atol=1e-15)
    m4 = np.einsum("l,lp,lq,lr,ls->pqrs", w, c, c, c, c)
    d = np.eye(3)
    iso = (np.einsum("pq,rs->pqrs", d, d) + np.einsum("pr,qs->pqrs", d, d) + np.einsum("ps,qr->pqrs", d, d)) / 9.0
    np.testing.assert_allclose(m4, iso, atol=1e-15)
    assert np.all(t["H3"][0] == 0.0)                      # H3 of the rest vector
    for l in range(nl):                                     # bounce pairs are opposite
        assert np.all(c[t["bounce"][l]] == -c[l])
    # solids pairs (l,l+1), l=2,4,.. (1-based) are the bounce pairs
    for l in range(1, nl - 1, 2):
        assert t["bounce"][l] == l + 1


def _cfg(nl, n=(5, 4, 3), **kw):
    return O.Config(n[0], n[1], n[2], nl, **kw)


@pytest.mark.parametrize("nl", [19, 27])
@pytest.mark.parametrize("ibgk", [2, 3])
def test_equilibrium_moments(nl, ibgk):
    c = _cfg(nl, ibgk=ibgk)
    o = O.Oracle(c, np.float64)
    rng = np.random.default_rng(3)
    rho = 1.0 + 0.05 * rng.uniform(-1, 1, c.sshape)
    u, v, w = (0.08 * rng.uniform(-1, 1, c.sshape) for _ in range(3))
    feq = o.zeros_f()
    o.fequil3(feq, rho, u, v, w)
    t = O.tables(nl, np.float64)
    cc = np.stack([t["cx"], t["cy"], t["cz"]], 1).astype(np.float64)
    s = (slice(1, -1),) * 3
    np.testing.assert_allclose(feq[s].sum(-1), rho[s], rtol=1e-14)
    vel = np.stack([u[s], v[s], w[s]], -1)
    np.testing.assert_allclose(feq[s] @ cc, rho[s][..., None] * vel, atol=1e-15)
    pi = np.einsum("...l,lp,lq->...pq", feq[s], cc, cc)
    expect = rho[s][..., None, None] * (np.eye(3) / 3.0 + vel[..., :, None] * vel[..., None, :])
    np.testing.assert_allclose(pi, expect, atol=1e-14)


@pytest.mark.parametrize("nl", [19, 27])
def test_regularized_equilibrium_is_zero(nl):
    c = _cfg(nl)
    o = O.Oracle(c, np.float64)
    rng = np.random.default_rng(5)
    rho = 1.0 + 0.05 * rng.uniform(-1, 1, c.sshape)
    u, v, w = (0.05 * rng.uniform(-1, 1, c.sshape) for _ in range(3))
    feq = o.zeros_f()
    o.fequil3(feq, rho, u, v, w)
    f = feq.copy()
    o.regularization(f, feq, u, v, w)
    assert np.abs(f).max() < 1e-16


@pytest.mark.parametrize("nl", [19, 27])
def test_uniform_flow_is_fixed_point(nl):
    """Periodic box at uniform equilibrium: fneq = 0 => nu_t = 0, drift permutes
    identical values, so f stays put (to round-off)."""
    c = _cfg(nl, n=(6, 5, 4), ibnd=0, jbnd=0, kbnd=0)
    o = O.Oracle(c, np.float64)
    rho = np.ones(c.sshape)
    u = np.full(c.sshape, 0.04)
    v = np.full(c.sshape, -0.01)
    w = np.full(c.sshape, 0.02)
    fA, fB = o.zeros_f(), o.zeros_f()
    o.init(fA, fB, rho, u, v, w, np.zeros(c.nz))
    f0 = fA.copy()
    tau = np.full(c.sshape, 3e-4 + 0.5)
    o.run(fA, fB, rho, u, v, w, tau, np.zeros(c.nz), 5)
    np.testing.assert_allclose(fA, f0, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(tau, 3e-4 + 0.5, rtol=1e-14)


@pytest.mark.parametrize("nl", [19, 27])
def test_periodic_mass_and_momentum_conservation(nl):
    c = _cfg(nl, n=(6, 5, 4), ibnd=0, jbnd=0, kbnd=0)
    o = O.Oracle(c, np.float64)
    rng = np.random.default_rng(11)
    s = (slice(1, -1),) * 3
    rho = np.ones(c.sshape)
    rho[s] += 0.01 * rng.uniform(-1, 1, rho[s].shape)
    u, v, w = (np.zeros(c.sshape) for _ in range(3))
    for a in (u, v, w):
        a[s] = 0.03 * rng.uniform(-1, 1, a[s].shape)
    fA, fB = o.zeros_f(), o.zeros_f()
    o.init(fA, fB, rho, u, v, w, np.zeros(c.nz))
    t = O.tables(nl, np.float64)
    cc = np.stack([t["cx"], t["cy"], t["cz"]], 1).astype(np.float64)
    m0, p0 = fA[s].sum(), (fA[s] @ cc).sum(axis=(0, 1, 2))
    tau = np.full(c.sshape, 3e-4 + 0.5)
    o.run(fA, fB, rho, u, v, w, tau, np.zeros(c.nz), 8)
    assert abs(fA[s].sum() - m0) < 1e-12 * abs(m0)
    np.testing.assert_allclose((fA[s] @ cc).sum(axis=(0, 1, 2)), p0, atol=1e-12)


@pytest.mark.parametrize("nl", [19, 27])
def test_drift_is_permutation(nl):
    c = _cfg(nl, n=(6, 5, 4), ibnd=0, jbnd=0, kbnd=0)
    o = O.Oracle(c, np.float64)
    rng = np.random.default_rng(2)
    f = rng.uniform(0, 1, c.fshape)
    f2 = o.zeros_f()
    o.boundarycond(f, f2, np.zeros(c.nz))     # periodic ghost fill of f
    out = o.zeros_f()
    o.drift(out, f)
    s = (slice(1, -1),) * 3
    for l in range(nl):
        np.testing.assert_array_equal(np.sort(out[s][..., l].ravel()), np.sort(f[s][..., l].ravel()))


@pytest.mark.parametrize("nl", [19, 27])
def test_solids_involution(nl):
    c = _cfg(nl)
    o = O.Oracle(c, np.float32)
    rng = np.random.default_rng(8)
    f = rng.uniform(0, 1, c.fshape).astype(np.float32)
    m = (rng.uniform(0, 1, c.sshape) < 0.5).astype(np.int32)
    g = f.copy()
    o.solids(g, m)
    assert not np.array_equal(g, f)
    o.solids(g, m)
    np.testing.assert_array_equal(g, f)


def test_vreman_zero_fneq_gives_molecular_tau():
    c = _cfg(27)
    o = O.Oracle(c, np.float32)
    rng = np.random.default_rng(1)
    rho = np.ones(c.sshape, np.float32)
    u, v, w = (0.05 * rng.uniform(-1, 1, c.sshape).astype(np.float32) for _ in range(3))
    feq = o.zeros_f()
    o.fequil3(feq, rho, u, v, w)
    tau = np.zeros(c.sshape, np.float32)
    f = feq.copy()
    o.postcoll(f, tau, rho, u, v, w)
    s = (slice(1, -1),) * 3
    # fneq is pure round-off here; nu_t must stay far below nu
    assert np.all(np.abs(tau[s] - np.float32(3 * 1e-4 + 0.5)) < 2e-4)


@pytest.mark.parametrize("nl", [19, 27])
def test_forcing_changes_momentum_by_minus_the_force(nl):
    """forcings_apply (m_forcings_apply_kernel.F90): sum df = 0 and sum c df = rho du = -F
    (second-order equilibria carry mass and momentum exactly); F = 0 changes nothing."""
    cfg = O.Config(6, 5, 4, nl)
    o = O.Oracle(cfg, np.float64)
    rng = np.random.default_rng(2)
    rho = 1.0 + 0.01 * rng.standard_normal(cfg.sshape)
    u, v, w = (0.03 * rng.standard_normal(cfg.sshape) for _ in range(3))
    f0 = rng.uniform(0.0, 0.1, cfg.fshape)
    F = 1e-4 * rng.standard_normal(cfg.sshape + (3,))
    f = f0.copy()
    o.forcings_apply(f, F, rho, u, v, w)
    t = O.tables(nl, np.float64)
    c = np.stack([t["cx"], t["cy"], t["cz"]], 1).astype(np.float64)
    inner = (slice(1, -1),) * 3
    df = (f - f0)[inner]
    np.testing.assert_allclose(df.sum(-1), 0.0, atol=1e-15)
    np.testing.assert_allclose(df @ c, -F[inner], rtol=1e-9, atol=1e-16)
    assert np.array_equal(f[0], f0[0])                     # ghost cells untouched
    g = f0.copy()
    o.forcings_apply(g, np.zeros_like(F), rho, u, v, w)
    assert np.array_equal(g, f0)


def test_oracle_results_do_not_depend_on_the_thread_count():
    """No oracle loop reduces across OpenMP threads, so the CPU baseline's thread
    count changes its speed, never its numbers: 1 and 4 threads agree bit for bit
    over a run with solids and the turbulence slice."""
    import numpy as np
    from lbm_b200 import workloads as W
    from oracle import oracle as O
    wl = W.Workload("threads", 20, 10, 8, 27, steps=4, sphere=(6, 5, 4, 2), lturb=True, ampl=1e-3, nrturb=3)
    cfg = O.Config(wl.nx, wl.ny, wl.nz, 27, iturb_pos=5, lsolids=True, lturb=True, nrturb=wl.nrturb, ampl=wl.ampl)
    blank = W.blanking(wl)
    turb = W.turbulence_fields(wl.ny, wl.nz, wl.nrturb, 3)
    import os
    before = O._threads
    outs = []
    try:
        for n in (1, 4):
            O.set_threads(n)
            o = O.Oracle(cfg, np.float32)
            rho, u, v, w = W.initial_macro(wl)
            uvel = W.inflow_profile(wl)
            fA, fB = o.zeros_f(), o.zeros_f()
            o.init(fA, fB, rho, u, v, w, uvel)
            tau = np.full(cfg.sshape, 3 * np.float32(1e-4) + 0.5, np.float32)
            o.run(fA, fB, rho, u, v, w, tau, uvel, wl.steps, blanking=blank, uu=turb[0], vv=turb[1], ww=turb[2])
            outs.append((fA, fB, rho, u, v, w))
    finally:
        O.set_threads(before if before else (os.cpu_count() or 1))
    for a, b in zip(*outs):
        assert np.array_equal(a.view(np.int32), b.view(np.int32))
