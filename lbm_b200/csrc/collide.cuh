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
// arithmetic is FP32 on offsets f' = f - w_l.
#pragma once

#include "common.cuh"

namespace lbm {

struct CollideParams {
    float kinevisc;   // nu
    float cvre;       // 2.5 * smagorinsky^2   (m_postcoll.F90:46)
    float eps;        // sqrt(tiny(1.0))       (m_postcoll.F90:47)
    float tau0;       // 3 nu + 0.5, the relaxation time without Vreman (main.F90:262)
    int ibgk, ihrr, ivreman;
};

// acc += coef * x for coef in {-1, 0, 1} known at compile time after unrolling
__device__ __forceinline__ void macc(float& acc, int coef, float x) {
    if (coef > 0) acc += x;
    else if (coef < 0) acc -= x;
}

struct Moments {
    float s0, jx, jy, jz, pxx, pyy, pzz, pxy, pxz, pyz;
};

template <int Q>
__device__ __forceinline__ Moments moments(const float (&fp)[Q]) {
    Moments m = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
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

__device__ __forceinline__ float cdot(int cx, int cy, int cz, float x, float y, float z) {
    float r = 0.f;
    macc(r, cx, x);
    macc(r, cy, y);
    macc(r, cz, z);
    return r;
}

// Turbulence increment du = ampl * (uu, vv, ww) at the forcing slice.
struct TurbIn {
    bool on;
    float dux, duy, duz;
};

// Collide one cell in place.  fp holds offsets f' = f - w_l on entry and the
// post-collision offsets (plus turbulence increment, solid swap) on exit.
//   drho = rho - 1, rho, u: the moments the collision uses (postcoll's rho,u,v,w)
//   s0, pi: sum f' and the raw second moments of the cell's own f'
//   tau_in: relaxation time used when ivreman == 0
// Returns the relaxation time tau of the cell.
template <int Q>
__device__ __forceinline__ float collide(float (&fp)[Q], const Moments& m, float drho, float rho, float ux, float uy,
                                         float uz, const CollideParams& cp, float abl, float tau_in, bool solid,
                                         const TurbIn& tb) {
    const float third = 1.0f / 3.0f;
    const float rux = rho * ux, ruy = rho * uy, ruz = rho * uz;
    const float axx = m.pxx - m.s0 * third - rux * ux;
    const float ayy = m.pyy - m.s0 * third - ruy * uy;
    const float azz = m.pzz - m.s0 * third - ruz * uz;
    const float axy = m.pxy - rux * uy;
    const float axz = m.pxz - rux * uz;
    const float ayz = m.pyz - ruy * uz;
    const float tr = axx + ayy + azz;

    float tau = tau_in;
    if (cp.ivreman) {
        // Vreman (2004) with alpha = a2 (see header); guards as m_postcoll_kernel.F90:270-299
        float amag = axx * axx + ayy * ayy + azz * azz + 2.0f * (axy * axy + axz * axz + ayz * ayz);
        amag = fmaxf(amag, 1.17549435e-38f);
        const float b11 = cp.eps + axx * axx + axy * axy + axz * axz;
        const float b22 = cp.eps + axy * axy + ayy * ayy + ayz * ayz;
        const float b33 = cp.eps + axz * axz + ayz * ayz + azz * azz;
        const float b12 = cp.eps + axx * axy + axy * ayy + axz * ayz;
        const float b13 = cp.eps + axx * axz + axy * ayz + axz * azz;
        const float b23 = cp.eps + axy * axz + ayy * ayz + ayz * azz;
        const float bb = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
        const float t = bb / amag;
        const float nut = (t > cp.eps) ? cp.cvre * sqrtf(t) : 0.0f;
        tau = 3.0f * (cp.kinevisc + nut + abl) + 0.5f;
    }
    const float K = 1.0f - 1.0f / tau;
    const bool cubic = (cp.ibgk == 3);
    const float usq = ux * ux + uy * uy + uz * uz;
    const float R45 = 4.5f * rho;
    const float R45o = cubic ? R45 : 0.0f;
    const float A0 = drho - 1.5f * rho * usq;              // even equilibrium part / w (cu = 0)
    const float B0 = 3.0f * rho - (cubic ? R45 * usq : 0.0f);  // odd equilibrium part / (w cu), cu^2 term aside

    // turbulence increment feq(rho, u + du) - feq(rho, u) (m_inflow_turbulence_forcing.F90:77-126)
    float dusq = 0.f;
    if (tb.on) dusq = tb.dux * (2.0f * ux + tb.dux) + tb.duy * (2.0f * uy + tb.duy) + tb.duz * (2.0f * uz + tb.duz);
    const float usq2 = usq + dusq;

    if (cp.ihrr) {
        const float C0 = A0 - 1.5f * K * tr;
        const float D0 = B0 - 4.5f * K * tr;
        const float K45 = 4.5f * K, K135 = 13.5f * K, K9 = 9.0f * K;
        const float bxy = 2.0f * axy, bxz = 2.0f * axz, byz = 2.0f * ayz;
        const float vx = axx * ux + axy * uy + axz * uz;
        const float vy = axy * ux + ayy * uy + ayz * uz;
        const float vz = axz * ux + ayz * uy + azz * uz;
        {
            float e = lat_w<Q>(0) * C0;
            if (tb.on) e += lat_w<Q>(0) * rho * (-1.5f * dusq);
            fp[0] = e;
        }
#pragma unroll
        for (int l = 1; l < Q; l += 2) {
            const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
            const float w = lat_w<Q>(l);
            const float cu = cdot(cx, cy, cz, ux, uy, uz);
            float cac = 0.f;
            macc(cac, cx * cx, axx);
            macc(cac, cy * cy, ayy);
            macc(cac, cz * cz, azz);
            macc(cac, cx * cy, bxy);
            macc(cac, cx * cz, bxz);
            macc(cac, cy * cz, byz);
            const float cau = cdot(cx, cy, cz, vx, vy, vz);
            const float cu2 = cu * cu;
            float E = w * (C0 + R45 * cu2 + K45 * cac);
            float O = w * (cu * (D0 + R45o * cu2 + K135 * cac) - K9 * cau);
            if (tb.on) {
                const float dcu = cdot(cx, cy, cz, tb.dux, tb.duy, tb.duz);
                const float cun = cu + dcu;
                E += w * rho * (4.5f * dcu * (2.0f * cu + dcu) - 1.5f * dusq);
                float od = 3.0f * dcu;
                if (cubic) od += 4.5f * dcu * (cun * cun + cun * cu + cu2 - usq2) - 4.5f * cu * dusq;
                O += w * rho * od;
            }
            if (solid) O = -O;
            fp[l] = E + O;
            fp[l + 1] = E - O;
        }
    } else {
        // plain BGK on the unregularized fneq: f' = (1-K) feq' + K f'
        const float omk = 1.0f - K;
        {
            float e = omk * lat_w<Q>(0) * A0 + K * fp[0];
            if (tb.on) e += lat_w<Q>(0) * rho * (-1.5f * dusq);
            fp[0] = e;
        }
#pragma unroll
        for (int l = 1; l < Q; l += 2) {
            const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
            const float w = lat_w<Q>(l);
            const float cu = cdot(cx, cy, cz, ux, uy, uz);
            const float cu2 = cu * cu;
            const float Eeq = w * (A0 + R45 * cu2);
            const float Oeq = w * cu * (B0 + R45o * cu2);
            float p = omk * (Eeq + Oeq) + K * fp[l];
            float q = omk * (Eeq - Oeq) + K * fp[l + 1];
            if (tb.on) {
                const float dcu = cdot(cx, cy, cz, tb.dux, tb.duy, tb.duz);
                const float cun = cu + dcu;
                const float dE = w * rho * (4.5f * dcu * (2.0f * cu + dcu) - 1.5f * dusq);
                float od = 3.0f * dcu;
                if (cubic) od += 4.5f * dcu * (cun * cun + cun * cu + cu2 - usq2) - 4.5f * cu * dusq;
                const float dO = w * rho * od;
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
