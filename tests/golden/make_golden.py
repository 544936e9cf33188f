"""Independent numpy restatement of the reference step + fixture generator.

The reference (geirev/LBM, Fortran/CUDA Fortran) ships no golden vectors and
cannot be built here, so these fixtures come from a second restatement of its
routines, written vectorised in numpy (float64) and independently of the C++
oracle.  Agreement between the two restatements pins the oracle's
transcription of the Fortran; each function cites the routine it restates.

Run from the repository root:  python tests/golden/make_golden.py
Output: tests/golden/golden_small.npz (a few hundred KB).
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "golden_small.npz")

# mod_D3Q27setup.F90:28-48 (1-based order kept; index 0 here is l=1 there)
C27 = np.array([
    [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1],
    [0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 0, 0, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1],
    [0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1]])
C19 = C27[:, :19]


def lattice(nl):
    c = (C19 if nl == 19 else C27).T.astype(np.int64)          # (nl, 3)
    s = np.abs(c).sum(1)
    if nl == 19:
        w = np.choose(s, [1 / 3, 1 / 18, 1 / 36])
    else:
        w = np.choose(s, [8 / 27, 2 / 27, 1 / 54, 1 / 216])
    cf = c.astype(np.float64)
    d = np.eye(3)
    H2 = np.einsum("lp,lq->lpq", cf, cf) - d[None] / 3.0
    H3 = (np.einsum("lp,lq,lr->lpqr", cf, cf, cf)
          - (np.einsum("lp,qr->lpqr", cf, d) + np.einsum("lq,pr->lpqr", cf, d) + np.einsum("lr,pq->lpqr", cf, d)) / 3.0)
    return c, w, H2, H3


def opposite(c, v):
    return int(np.nonzero((c == np.asarray(v)).all(1))[0][0])


# ---- per-cell algebra (arrays: scalars (...), vel (...,3), f (..., nl)) ------
def feq_cells(lat, rho, vel, ibgk, rest_h3=False):
    """fequil3_kernel (m_fequil3_kernel.F90:58-113); rest_h3 selects the
    fequil3_block_kernel variant that adds H3 for every l (:273-283)."""
    c, w, H2, H3 = lat
    A2 = 4.5 * rho[..., None, None] * vel[..., :, None] * vel[..., None, :]
    cu = vel @ c.T.astype(np.float64)
    t = rho[..., None] * (1.0 + 3.0 * cu) + np.einsum("lpq,...pq->...l", H2, A2)
    if ibgk == 3:
        A3 = A2[..., None] * vel[..., None, None, :]
        h3 = np.einsum("lpqr,...pqr->...l", H3, A3)
        if not rest_h3:
            h3[..., 0] = 0.0
        t = t + h3
    return w * t


def regularize_cells(lat, fneq, vel):
    """R(fneq) as in m_postcoll_kernel.F90:189-244 / m_regularization_kernel.F90:44-114."""
    c, w, H2, H3 = lat
    a2 = np.einsum("lpq,...l->...pq", H2, fneq)
    a3 = (vel[..., :, None, None] * a2[..., None, :, :] + vel[..., None, :, None] * np.swapaxes(a2, -1, -2)[..., :, None, :]
          + vel[..., None, None, :] * a2[..., :, :, None])
    return w * (np.einsum("lpq,...pq->...l", H2, 4.5 * a2) + np.einsum("lpqr,...pqr->...l", H3, 4.5 * a3))


def vreman_tau(lat, fneq, kinevisc, smag, ablk, standalone=False):
    """Vreman nu_t: m_postcoll_kernel.F90:189-239 or m_vreman_kernel.F90:47-91."""
    c, w, H2, H3 = lat
    alpha = np.einsum("lpq,...l->...pq", H2, fneq)
    eps = np.sqrt(np.finfo(np.float64).tiny)
    off = 1e-5 if standalone else 0.0
    amag = off + (alpha ** 2).sum((-1, -2))
    if not standalone:
        amag = np.maximum(amag, np.finfo(np.float64).tiny)
    beta = (eps if not standalone else 1e-5) + np.einsum("...mp,...mq->...pq", alpha, alpha)
    B = (beta[..., 0, 0] * beta[..., 1, 1] - beta[..., 0, 1] ** 2 + beta[..., 0, 0] * beta[..., 2, 2]
         - beta[..., 0, 2] ** 2 + beta[..., 1, 1] * beta[..., 2, 2] - beta[..., 1, 2] ** 2)
    t = B / amag
    nut = np.where(t > eps, 2.5 * smag ** 2 * np.sqrt(np.maximum(t, 0.0)), 0.0)
    return 3.0 * (kinevisc + nut + ablk) + 0.5


# ---- grid routines on f[k, j, i, l] (ghost-inclusive) -----------------------
def interior(a):
    return a[1:-1, 1:-1, 1:-1]


def postcoll(lat, f, tau, rho, u, v, w, cfg):
    vel = np.stack([interior(u), interior(v), interior(w)], -1)
    r = interior(rho)
    fe = feq_cells(lat, r, vel, cfg["ibgk"])
    fneq = interior(f) - fe
    if cfg["ihrr"] == 1:
        fneq = regularize_cells(lat, fneq, vel)
    if cfg["ivreman"] == 1:
        abl = np.zeros(f.shape[0] - 2)[:, None, None]
        tau[1:-1, 1:-1, 1:-1] = vreman_tau(lat, fneq, cfg["kinevisc"], cfg["smagorinsky"], abl)
    fac = 1.0 - 1.0 / interior(tau)
    f[1:-1, 1:-1, 1:-1] = fe + fac[..., None] * fneq


def drift(lat, fout, fin):
    """m_drift_kernel.F90:42: fout(l,x) = fin(l, x - c_l), interior x."""
    c = lat[0]
    nz, ny, nx = (s - 2 for s in fin.shape[:3])
    for l in range(c.shape[0]):
        cx, cy, cz = c[l]
        fout[1:-1, 1:-1, 1:-1, l] = fin[1 - cz:nz + 1 - cz, 1 - cy:ny + 1 - cy, 1 - cx:nx + 1 - cx, l]


def macrovars(lat, f):
    c = lat[0].astype(np.float64)
    rho = f.sum(-1)
    return rho, (f @ c[:, 0]) / rho, (f @ c[:, 1]) / rho, (f @ c[:, 2]) / rho


def closed(lat, f1, f2, axis, plane, ghost, opt):
    """boundary_{i,j,k}_closed_kernel: axis 0=i,1=j,2=k; plane 1 or n."""
    c = lat[0]
    shp = f1.shape[:3][::-1]  # (nx+2, ny+2, nz+2)
    n = shp[axis] - 2
    for l in range(c.shape[0]):
        cl = c[l]
        if not ((plane == 1 and cl[axis] < 0) or (plane == n and cl[axis] > 0)):
            continue
        mv = opt * cl.copy()
        mv[axis] = -cl[axis]
        m = opposite(c, mv)
        # tangential ranges 1..n of the other two axes, ghost plane on `axis`
        sl_g = [slice(1, -1)] * 3
        sl_g[axis] = ghost
        kz, jy, ix = sl_g[2], sl_g[1], sl_g[0]
        f1[kz, jy, ix, m] = f2[kz, jy, ix, l]
        src = []
        for a in range(3):
            if a == axis:
                src.append(plane)
            else:
                na = shp[a] - 2
                src.append(slice(1 - cl[a], na + 1 - cl[a]))
        f1[kz, jy, ix, l] = f1[src[2], src[1], src[0], l]


def inflow(lat, f, uvel, rho0, udir):
    c, w = lat[0], lat[1]
    pi = 3.1415927410125732
    uu = uvel[:, None]
    ux = uu * np.cos(udir * pi / 180.0)
    uy = uu * np.sin(udir * pi / 180.0)
    fg = f[1:-1, 1:-1, 1, :] - 2.0 * w * rho0 * (c[:, 0] * ux[..., None] + c[:, 1] * uy[..., None]) * 3.0
    for l in range(c.shape[0]):
        if c[l, 0] <= 0:
            f[1:-1, 1:-1, 0, l] = fg[..., l]
        else:
            f[1:-1, 1:-1, 0, l] = fg[..., opposite(c, -c[l])]
    f[1:-1, 1:-1, -1, :] = f[1:-1, 1:-1, -2, :]


def edges_jk(lat, f1, f2, opt):
    c = lat[0]
    ny, nz = f1.shape[1] - 2, f1.shape[0] - 2
    for (jg, kg, sy, sz, ji, ki, useopt) in [(0, 0, -1, -1, 1, 1, 1), (ny + 1, 0, 1, -1, ny, 1, 1),
                                              (0, nz + 1, -1, 1, 1, nz, 1), (ny + 1, nz + 1, 1, 1, ny, nz, 0)]:
        ls = [l for l in range(c.shape[0]) if c[l, 1] * sy > 0 and c[l, 2] * sz > 0]
        for l in ls:
            m = opposite(c, [(opt if useopt else 1) * c[l, 0], -c[l, 1], -c[l, 2]])
            f1[kg, jg, 1:-1, m] = f2[kg, jg, 1:-1, l]
        for l in ls:
            f1[kg, jg, 1:-1, l] = f1[ki, ji, 1:-1, l]


def edges_ij(lat, f1, f2, opt):
    c = lat[0]
    nx, ny = f1.shape[2] - 2, f1.shape[1] - 2
    for (ig, jg, sx, sy, ii, ji) in [(0, 0, -1, -1, 1, 1), (nx + 1, 0, 1, -1, nx, 1),
                                     (0, ny + 1, -1, 1, 1, ny), (nx + 1, ny + 1, 1, 1, nx, ny)]:
        ls = [l for l in range(c.shape[0]) if c[l, 0] * sx > 0 and c[l, 1] * sy > 0]
        for l in ls:
            f1[1:-1, jg, ig, opposite(c, [-c[l, 0], -c[l, 1], opt * c[l, 2]])] = f2[1:-1, jg, ig, l]
        for l in ls:
            f1[1:-1, jg, ig, l] = f1[1:-1, ji, ii, l]


def edges_ik(lat, f1, f2, opt):
    c = lat[0]
    nx, nz = f1.shape[2] - 2, f1.shape[0] - 2
    for (ig, kg, sx, sz, ii, ki) in [(0, 0, -1, -1, 1, 1), (nx + 1, 0, 1, -1, nx, 1),
                                     (0, nz + 1, -1, 1, 1, nz), (nx + 1, nz + 1, 1, 1, nx, nz)]:
        ls = [l for l in range(c.shape[0]) if c[l, 0] * sx > 0 and c[l, 2] * sz > 0]
        for l in ls:
            f1[kg, 1:-1, ig, opposite(c, [-c[l, 0], opt * c[l, 1], -c[l, 2]])] = f2[kg, 1:-1, ig, l]
        for l in ls:
            f1[kg, 1:-1, ig, l] = f1[ki, 1:-1, ii, l]


def corners(lat, f1, f2, opt):
    c = lat[0]
    nx, ny, nz = f1.shape[2] - 2, f1.shape[1] - 2, f1.shape[0] - 2
    for ic in (0, nx + 1):
        for jc in (0, ny + 1):
            for kc in (0, nz + 1):
                sg = np.array([-1 if ic == 0 else 1, -1 if jc == 0 else 1, -1 if kc == 0 else 1])
                ls = [l for l in range(c.shape[0]) if (c[l] * sg > 0).all()]
                for l in ls:
                    f1[kc, jc, ic, opposite(c, opt * c[l])] = f2[kc, jc, ic, l]
                for l in ls:
                    f1[kc, jc, ic, l] = f1[kc - c[l, 2], jc - c[l, 1], ic - c[l, 0], l]


def opts(code):
    return {11: (-1, -1), 12: (-1, 1), 21: (1, -1), 22: (1, 1)}.get(code, (0, 0))


def boundarycond(lat, f1, f2, uvel, cfg):
    """m_boundarycond.F90:14-468 in its dispatch order."""
    ib, jb, kb = cfg["ibnd"], cfg["jbnd"], cfg["kbnd"]
    nx, ny, nz = f1.shape[2] - 2, f1.shape[1] - 2, f1.shape[0] - 2

    def per():
        if ib == 0:
            f1[:, :, 0] = f1[:, :, nx]
            f1[:, :, nx + 1] = f1[:, :, 1]
        if jb == 0:
            f1[:, 0] = f1[:, ny]
            f1[:, ny + 1] = f1[:, 1]
        if kb == 0:
            f1[0] = f1[nz]
            f1[nz + 1] = f1[1]
    per()
    for axis, code, n in ((0, ib, nx), (1, jb, ny), (2, kb, nz)):
        o1, oN = opts(code)
        if o1 != 0:
            closed(lat, f1, f2, axis, 1, 0, o1)
            closed(lat, f1, f2, axis, n, n + 1, oN)
    if jb > 10 and kb > 10:
        edges_jk(lat, f1, f2, 1 if (jb == 22 and kb == 22) else -1)
    if ib > 10 and jb > 10:
        edges_ij(lat, f1, f2, 1 if (ib == 22 and jb == 22) else -1)
    if ib > 10 and kb > 10:
        edges_ik(lat, f1, f2, 1 if (ib == 22 and kb == 22) else -1)
    if ib > 10 and jb > 10 and kb > 10:
        corners(lat, f1, f2, -1)
    if ib == 1:
        inflow(lat, f1, uvel, cfg["rho0"], cfg["udir"])
    per()


def solids(f, blank):
    m = interior(blank) != 0
    fi = f[1:-1, 1:-1, 1:-1]
    nl = f.shape[-1]
    for l in range(1, nl - 1, 2):
        a = fi[..., l][m].copy()
        fi[..., l][m] = fi[..., l + 1][m]
        fi[..., l + 1][m] = a


def fillghosts(f):
    nz, ny, nx = (s - 2 for s in f.shape[:3])
    k = np.clip(np.arange(nz + 2), 1, nz)
    j = np.clip(np.arange(ny + 2), 1, ny)
    i = np.clip(np.arange(nx + 2), 1, nx)
    return f[k][:, j][:, :, i].copy()


def turb_df(lat, rho, u, v, w, uu, vv, ww, it, cfg):
    """m_inflow_turbulence_forcing.F90:44-128; returns df[k,j,l] (ny,nz interior)."""
    ip = cfg["iturb_pos"]
    nrt = cfg["nrturb"]
    lit = it % nrt or nrt
    r = rho[1:-1, 1:-1, ip]
    vel = np.stack([u[1:-1, 1:-1, ip], v[1:-1, 1:-1, ip], w[1:-1, 1:-1, ip]], -1)
    f1 = feq_cells(lat, r, vel, cfg["ibgk"], rest_h3=True)
    a = cfg["ampl"]
    vel2 = vel + a * np.stack([uu[lit], vv[lit], ww[lit]], -1)
    f2 = feq_cells(lat, r, vel2, cfg["ibgk"], rest_h3=True)
    return f2 - f1


def init(lat, rho, u, v, w, uvel, cfg):
    """main.F90:243-247."""
    vel = np.stack([interior(u), interior(v), interior(w)], -1)
    fB = np.zeros(rho.shape + (lat[0].shape[0],))
    fB[1:-1, 1:-1, 1:-1] = feq_cells(lat, interior(rho), vel, cfg["ibgk"])
    fB = fillghosts(fB)
    fA = fB.copy()
    boundarycond(lat, fB, fA, uvel, cfg)
    boundarycond(lat, fA, fB, uvel, cfg)
    return fA, fB


def run(lat, fA, fB, rho, u, v, w, tau, uvel, nsteps, cfg, blank=None, turb=None):
    """main.F90:283-329.  Returns (f1, f2, rho, u, v, w, tau)."""
    f1, f2 = fA, fB
    for it in range(1, nsteps + 1):
        if turb is not None:
            df = turb_df(lat, rho, u, v, w, *turb, it, cfg)
        postcoll(lat, f1, tau, rho, u, v, w, cfg)
        if turb is not None:
            f1[1:-1, 1:-1, cfg["iturb_pos"], :] += df
        if blank is not None:
            solids(f1, blank)
        boundarycond(lat, f1, f2, uvel, cfg)
        drift(lat, f2, f1)
        f1, f2 = f2, f1
        rho, u, v, w = macrovars(lat, f1)
    return f1, f2, rho, u, v, w, tau


# ---- fixture generation ------------------------------------------------------
BASE = dict(ibgk=3, ihrr=1, ivreman=1, ibnd=1, jbnd=0, kbnd=12, iturb_pos=3, nrturb=4,
            kinevisc=1e-4, smagorinsky=0.15, rho0=1.0, udir=0.0, ampl=1e-2)


def physical_state(rng, lat, nx, ny, nz, noise):
    shp = (nz + 2, ny + 2, nx + 2)
    rho = 1.0 + 0.01 * rng.uniform(-1, 1, shp)
    u = 0.05 + noise * rng.uniform(-1, 1, shp)
    v = noise * rng.uniform(-1, 1, shp)
    w = noise * rng.uniform(-1, 1, shp)
    vel = np.stack([u, v, w], -1)
    f = feq_cells(lat, rho, vel, 3)
    f = f * (1.0 + 0.02 * rng.uniform(-1, 1, f.shape))     # add non-equilibrium
    return tuple(a.astype(np.float32).astype(np.float64) for a in (f, rho, u, v, w))


def main():
    out = {}
    nx, ny, nz = 4, 3, 3
    for nl in (19, 27):
        lat = lattice(nl)
        rng = np.random.default_rng(1000 + nl)
        f, rho, u, v, w = physical_state(rng, lat, nx, ny, nz, 0.02)
        p = "q%d_" % nl
        out[p + "f"], out[p + "rho"], out[p + "u"], out[p + "v"], out[p + "w"] = f, rho, u, v, w
        # fequil3
        feq = np.zeros_like(f)
        vel = np.stack([interior(u), interior(v), interior(w)], -1)
        feq[1:-1, 1:-1, 1:-1] = feq_cells(lat, interior(rho), vel, 3)
        out[p + "fequil3"] = feq
        feq2 = np.zeros_like(f)
        feq2[1:-1, 1:-1, 1:-1] = feq_cells(lat, interior(rho), vel, 2)
        out[p + "fequil2"] = feq2
        # postcoll variants
        for ihrr in (0, 1):
            for ivr in (0, 1):
                cfg = dict(BASE, ihrr=ihrr, ivreman=ivr)
                ff = f.copy()
                tau = np.full(rho.shape, 3 * 1e-4 + 0.5)
                postcoll(lat, ff, tau, rho, u, v, w, cfg)
                out[p + "postcoll_h%d_v%d_f" % (ihrr, ivr)] = ff
                out[p + "postcoll_h%d_v%d_tau" % (ihrr, ivr)] = tau
        # drift, macrovars
        fd = np.zeros_like(f)
        drift(lat, fd, f)
        out[p + "drift"] = fd
        r2, u2, v2, w2 = macrovars(lat, f)
        out[p + "macro"] = np.stack([r2, u2, v2, w2])
        # standalone regularization / vreman
        fr = f.copy()
        fr[1:-1, 1:-1, 1:-1] = regularize_cells(lat, interior(f) - interior(feq), vel)
        out[p + "regularization"] = fr
        fneq = f - feq
        tau = np.zeros(rho.shape)
        tau[1:-1, 1:-1, 1:-1] = vreman_tau(lat, interior(fneq), 1e-4, 0.15, 0.0, standalone=True)
        out[p + "vreman_in"] = fneq
        out[p + "vreman_tau"] = tau
        # boundary conditions: several codes on random (non-physical) f1, f2
        f1 = rng.uniform(0.0, 1.0, f.shape).astype(np.float32).astype(np.float64)
        f2 = rng.uniform(0.0, 1.0, f.shape).astype(np.float32).astype(np.float64)
        uvel = (0.05 + 0.01 * rng.uniform(-1, 1, nz)).astype(np.float32).astype(np.float64)
        out[p + "bc_f1"], out[p + "bc_f2"], out[p + "bc_uvel"] = f1, f2, uvel
        for (ib, jb, kb) in [(1, 0, 12), (0, 0, 0), (11, 22, 12), (22, 21, 11), (12, 11, 22), (1, 11, 22)]:
            cfg = dict(BASE, ibnd=ib, jbnd=jb, kbnd=kb, udir=10.0 if ib == 1 else 0.0)
            a, b = f1.copy(), f2.copy()
            boundarycond(lat, a, b, uvel, cfg)
            out[p + "bc_%d_%d_%d" % (ib, jb, kb)] = a
        # solids + fillghosts
        blank = (rng.uniform(0, 1, rho.shape) < 0.3).astype(np.int32)
        fs = f.copy()
        solids(fs, blank)
        out[p + "solids_mask"], out[p + "solids"] = blank, fs
        out[p + "fillghosts"] = fillghosts(f)
        # turbulence forcing slice
        nrt = BASE["nrturb"]
        uu, vv, ww = (rng.standard_normal((nrt + 1, nz, ny)).astype(np.float32).astype(np.float64) for _ in range(3))
        out[p + "turb_uu"], out[p + "turb_vv"], out[p + "turb_ww"] = uu, vv, ww
        out[p + "turb_df_it7"] = turb_df(lat, rho, u, v, w, uu, vv, ww, 7, BASE)
        # full run: init + 6 steps with a sphere-like mask and turbulence
        mx, my, mz = 6, 4, 4
        rng2 = np.random.default_rng(77 + nl)
        shp = (mz + 2, my + 2, mx + 2)
        rho0 = np.zeros(shp)
        u0 = np.zeros(shp)
        v0 = np.zeros(shp)
        w0 = np.zeros(shp)
        rho0[1:-1, 1:-1, 1:-1] = 1.0
        u0[1:-1, 1:-1, 1:-1] = (0.05 + 1e-3 * rng2.uniform(-1, 1, (mz, my, mx))).astype(np.float32)
        v0[1:-1, 1:-1, 1:-1] = (1e-3 * rng2.uniform(-1, 1, (mz, my, mx))).astype(np.float32)
        w0[1:-1, 1:-1, 1:-1] = (1e-3 * rng2.uniform(-1, 1, (mz, my, mx))).astype(np.float32)
        k3, j3, i3 = np.meshgrid(np.arange(mz + 2), np.arange(my + 2), np.arange(mx + 2), indexing="ij")
        blank2 = (((i3 - 4) ** 2 + (j3 - 2) ** 2 + (k3 - 2) ** 2) < 3).astype(np.int32)
        uvel2 = np.full(mz, np.float32(0.05), np.float64)
        uu2, vv2, ww2 = (rng2.standard_normal((nrt + 1, mz, my)).astype(np.float32).astype(np.float64) for _ in range(3))
        cfg = dict(BASE)
        fA, fB = init(lat, rho0, u0, v0, w0, uvel2, cfg)
        out[p + "run_init_fA"], out[p + "run_init_fB"] = fA.copy(), fB.copy()
        tau0 = np.full(shp, 3 * 1e-4 + 0.5)
        r1 = run(lat, fA.copy(), fB.copy(), rho0.copy(), u0.copy(), v0.copy(), w0.copy(), tau0.copy(),
                 uvel2, 6, cfg, blank=blank2, turb=(uu2, vv2, ww2))
        for name, arr in zip(("f1", "f2", "rho", "u", "v", "w", "tau"), r1):
            out[p + "run_" + name] = arr
        out[p + "run_in"] = np.stack([rho0, u0, v0, w0])
        out[p + "run_mask"] = blank2
        out[p + "run_uvel"] = uvel2
        out[p + "run_turb"] = np.stack([uu2, vv2, ww2])
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
