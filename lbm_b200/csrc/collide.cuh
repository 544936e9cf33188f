// collide.cuh -- closed-form collision of one cell (device code).
//
// Restates postcoll_kernel (m_postcoll_kernel.F90:7-255) without its dense
// tensor loops.  With H2_l = c c - I/3 and H3_l the third-order Hermite
// tensor (mod_D3Q27setup.F90:127-150), and u = (ux,uy,uz), cu = c.u:
//
//   feq_l  = w_l rho [1 + 3 cu + 4.5 cu^2 - 1.5 u^2 + 4.5 (cu^3 - cu u^2)]
//            (the cubic bracket is H3_l : A3 with A3 = 4.5 rho u u u, ibgk = 3)
//   a2     = sum_l H2_l (f_l - feq_l)
//          = Pi - I S0/3 - rho u u        (Pi = sum c c f', S0 = sum f', f' = f - w)
//   R(fneq)_l = 4.5 w_l [c.a2.c - tr/3 + cu (3 c.a2.c - tr) - 2 c.a2.u]
//            (H2_l:a2 and H3_l:A3 with A3 = u a2 + a2 u + ... , :189-244)
//   alpha  = sum_l H2_l R(fneq)_l = a2    (fourth-order isotropy of the lattice:
//            sum_l w_l H2_l H2_l = (1/9)(d d + d d), odd moments vanish)
//
// so the Vreman model (:255-304) works on a2 directly.  Directions c and -c
// share the even part E and flip the odd part O, so each opposite pair costs
// one evaluation: f'(+c) = E + O, f'(-c) = E - O.  The solid swap of
// m_solids.F90:28-32 exchanges exactly these pairs, i.e. negates O.  All
// arithmetic is on offsets f' = f - w_l in the type R: FP32 (the reference's
// default build) or FP64 (its DP build, where -r8 promotes every real).
#pragma once

#include "common.cuh"

namespace lbm {

template <typename R>
struct CollideParamsT {
    R kinevisc;       // nu
    R cvre;           // 2.5 * smagorinsky^2   (m_postcoll.F90:46)
    R eps;            // sqrt(tiny(1.0))       (m_postcoll.F90:47)
    R tau0;           // 3 nu + 0.5, the relaxation time without Vreman (main.F90:262)
    int ibgk, ihrr, ivreman;
};
using CollideParams = CollideParamsT<float>;

// acc += coef * x for coef in {-1, 0, 1} known at compile time after unrolling
__device__ __forceinline__ void macc(float& acc, int coef, float x) {
    if (coef > 0) acc += x;
    else if (coef < 0) acc -= x;
}
__device__ __forceinline__ void macc(double& acc, int coef, double x) {
    if (coef > 0) acc += x;
    else if (coef < 0) acc -= x;
}

template <typename R>
struct MomentsT {
    R s0, jx, jy, jz, pxx, pyy, pzz, pxy, pxz, pyz;
};
using Moments = MomentsT<float>;

template <int Q, typename R>
__device__ __forceinline__ MomentsT<R> moments(const R (&fp)[Q]) {
    MomentsT<R> m = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
        m.s0 += fp[l];
        macc(m.jx, cx, fp[l]);
        macc(m.jy, cy, fp[l]);
        macc(m.jz, cz, fp[l]);
        macc(m.pxx, cx * cx, fp[l]);
        macc(m.pyy, cy * cy, fp[l]);
        macc(m.pzz, cz * cz, fp[l]);
        macc(m.pxy, cx * cy, fp[l]);
        macc(m.pxz, cx * cz, fp[l]);
        macc(m.pyz, cy * cz, fp[l]);
    }
    return m;
}

template <typename R>
__device__ __forceinline__ R cdot(int cx, int cy, int cz, R x, R y, R z) {
    R r = R(0);
    macc(r, cx, x);
    macc(r, cy, y);
    macc(r, cz, z);
    return r;
}

// Turbulence increment du = ampl * (uu, vv, ww) at the forcing slice.
template <typename R>
struct TurbInT {
    bool on;
    R dux, duy, duz;
};
using TurbIn = TurbInT<float>;

// Collide one cell in place.  fp holds offsets f' = f - w_l on entry and the
// post-collision offsets (plus turbulence increment, solid swap) on exit.
//   drho = rho - 1, rho, u: the moments the collision uses (postcoll's rho,u,v,w)
//   s0, pi: sum f' and the raw second moments of the cell's own f'
//   tau_in: relaxation time used when ivreman == 0
// Returns the relaxation time tau of the cell.
template <int Q, typename R>
__device__ __forceinline__ R collide(R (&fp)[Q], const MomentsT<R>& m, R drho, R rho, R ux, R uy, R uz,
                                     const CollideParamsT<R>& cp, R abl, R tau_in, bool solid, const TurbInT<R>& tb) {
    const R third = R(1.0) / R(3.0);
    const R rux = rho * ux, ruy = rho * uy, ruz = rho * uz;
    const R axx = m.pxx - m.s0 * third - rux * ux;
    const R ayy = m.pyy - m.s0 * third - ruy * uy;
    const R azz = m.pzz - m.s0 * third - ruz * uz;
    const R axy = m.pxy - rux * uy;
    const R axz = m.pxz - rux * uz;
    const R ayz = m.pyz - ruy * uz;
    const R tr = axx + ayy + azz;

    R tau = tau_in;
    if (cp.ivreman) {
        // Vreman (2004) with alpha = a2 (see header); guards as m_postcoll_kernel.F90:204-233
        R amag = axx * axx + ayy * ayy + azz * azz + R(2.0) * (axy * axy + axz * axz + ayz * ayz);
        amag = real_max(amag, lat_tiny<R>());
        const R b11 = cp.eps + axx * axx + axy * axy + axz * axz;
        const R b22 = cp.eps + axy * axy + ayy * ayy + ayz * ayz;
        const R b33 = cp.eps + axz * axz + ayz * ayz + azz * azz;
        const R b12 = cp.eps + axx * axy + axy * ayy + axz * ayz;
        const R b13 = cp.eps + axx * axz + axy * ayz + axz * azz;
        const R b23 = cp.eps + axy * axz + ayy * ayz + ayz * azz;
        const R bb = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
        const R t = bb / amag;
        const R nut = (t > cp.eps) ? cp.cvre * real_sqrt(t) : R(0.0);
        tau = R(3.0) * (cp.kinevisc + nut + abl) + R(0.5);
    }
    const R K = R(1.0) - R(1.0) / tau;
    const bool cubic = (cp.ibgk == 3);
    const R usq = ux * ux + uy * uy + uz * uz;
    const R R45 = R(4.5) * rho;
    const R R45o = cubic ? R45 : R(0.0);
    const R A0 = drho - R(1.5) * rho * usq;              // even equilibrium part / w (cu = 0)
    const R B0 = R(3.0) * rho - (cubic ? R45 * usq : R(0.0));  // odd equilibrium part / (w cu), cu^2 term aside

    // turbulence increment feq(rho, u + du) - feq(rho, u) (m_inflow_turbulence_forcing.F90:77-126)
    R dusq = R(0);
    if (tb.on) dusq = tb.dux * (R(2.0) * ux + tb.dux) + tb.duy * (R(2.0) * uy + tb.duy) + tb.duz * (R(2.0) * uz + tb.duz);
    const R usq2 = usq + dusq;

    if (cp.ihrr) {
        const R C0 = A0 - R(1.5) * K * tr;
        const R D0 = B0 - R(4.5) * K * tr;
        const R K45 = R(4.5) * K, K135 = R(13.5) * K, K9 = R(9.0) * K;
        const R bxy = R(2.0) * axy, bxz = R(2.0) * axz, byz = R(2.0) * ayz;
        const R vx = axx * ux + axy * uy + axz * uz;
        const R vy = axy * ux + ayy * uy + ayz * uz;
        const R vz = axz * ux + ayz * uy + azz * uz;
        {
            R e = lat_w<Q, R>(0) * C0;
            if (tb.on) e += lat_w<Q, R>(0) * rho * (-R(1.5) * dusq);
            fp[0] = e;
        }
#pragma unroll
        for (int l = 1; l < Q; l += 2) {
            const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
            const R w = lat_w<Q, R>(l);
            const R cu = cdot(cx, cy, cz, ux, uy, uz);
            R cac = R(0);
            macc(cac, cx * cx, axx);
            macc(cac, cy * cy, ayy);
            macc(cac, cz * cz, azz);
            macc(cac, cx * cy, bxy);
            macc(cac, cx * cz, bxz);
            macc(cac, cy * cz, byz);
            const R cau = cdot(cx, cy, cz, vx, vy, vz);
            const R cu2 = cu * cu;
            R E = w * (C0 + R45 * cu2 + K45 * cac);
            R O = w * (cu * (D0 + R45o * cu2 + K135 * cac) - K9 * cau);
            if (tb.on) {
                const R dcu = cdot(cx, cy, cz, tb.dux, tb.duy, tb.duz);
                const R cun = cu + dcu;
                E += w * rho * (R(4.5) * dcu * (R(2.0) * cu + dcu) - R(1.5) * dusq);
                R od = R(3.0) * dcu;
                if (cubic) od += R(4.5) * dcu * (cun * cun + cun * cu + cu2 - usq2) - R(4.5) * cu * dusq;
                O += w * rho * od;
            }
            if (solid) O = -O;
            fp[l] = E + O;
            fp[l + 1] = E - O;
        }
    } else {
        // plain BGK on the unregularized fneq: f' = (1-K) feq' + K f'
        const R omk = R(1.0) - K;
        {
            R e = omk * lat_w<Q, R>(0) * A0 + K * fp[0];
            if (tb.on) e += lat_w<Q, R>(0) * rho * (-R(1.5) * dusq);
            fp[0] = e;
        }
#pragma unroll
        for (int l = 1; l < Q; l += 2) {
            const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
            const R w = lat_w<Q, R>(l);
            const R cu = cdot(cx, cy, cz, ux, uy, uz);
            const R cu2 = cu * cu;
            const R Eeq = w * (A0 + R45 * cu2);
            const R Oeq = w * cu * (B0 + R45o * cu2);
            R p = omk * (Eeq + Oeq) + K * fp[l];
            R q = omk * (Eeq - Oeq) + K * fp[l + 1];
            if (tb.on) {
                const R dcu = cdot(cx, cy, cz, tb.dux, tb.duy, tb.duz);
                const R cun = cu + dcu;
                const R dE = w * rho * (R(4.5) * dcu * (R(2.0) * cu + dcu) - R(1.5) * dusq);
                R od = R(3.0) * dcu;
                if (cubic) od += R(4.5) * dcu * (cun * cun + cun * cu + cu2 - usq2) - R(4.5) * cu * dusq;
                const R dO = w * rho * od;
                p += dE + dO;
                q += dE - dO;
            }
            if (solid) {
                fp[l] = q;
                fp[l + 1] = p;
            } else {
                fp[l] = p;
                fp[l + 1] = q;
            }
        }
    }
    return tau;
}

}  // namespace lbm
