// collide_rows.cuh -- the regularized collision of collide.cuh reorganised by
// lattice rows, for the steady fused step.
//
// Same equations as collide() (see collide.cuh), evaluated with shared partial
// sums.  The Q directions are grouped into the nine rows (cy, cz); a row holds
// the directions cx = -1, 0, +1 that the lattice has.  Every moment is a
// signed sum of three row sums (A = sum over cx, X = f(+1) - f(-1),
// B = f(+1) + f(-1)), and in the emission the scalar products c.u, c.a2.c
// and c.a2.u of the three directions of a row share their (cy, cz) part.
// The opposite of row (cy, cz) is row (-cy, -cz), so each row pair emits three
// opposite-direction pairs (one for the rows of D3Q19 without cx = +-1).
#pragma once

#include "collide.cuh"

namespace lbm {

template <int Q, int CY, int CZ>
struct Row {
    static constexpr int l0 = lat_find<Q>(0, CY, CZ);
    static constexpr int lp = lat_find<Q>(1, CY, CZ);
    static constexpr int lm = lat_find<Q>(-1, CY, CZ);
    static constexpr bool hasx = lp >= 0;
};

struct RowSum {
    float A, X, B;
};

template <int Q, int CY, int CZ>
__device__ __forceinline__ RowSum row_sum(const float (&f)[Q]) {
    using R = Row<Q, CY, CZ>;
    RowSum s;
    if constexpr (R::hasx) {
        s.B = f[R::lp] + f[R::lm];
        s.X = f[R::lp] - f[R::lm];
        s.A = s.B + f[R::l0];
    } else {
        s.B = 0.f;
        s.X = 0.f;
        s.A = f[R::l0];
    }
    return s;
}

// Moments of f' (sums of f - w_l, or of a scaled copy): same quantities as moments()
template <int Q>
__device__ __forceinline__ Moments moments_rows(const float (&f)[Q]) {
    const RowSum mm = row_sum<Q, -1, -1>(f), m0 = row_sum<Q, -1, 0>(f), mp = row_sum<Q, -1, 1>(f);
    const RowSum om = row_sum<Q, 0, -1>(f), oo = row_sum<Q, 0, 0>(f), op = row_sum<Q, 0, 1>(f);
    const RowSum pm = row_sum<Q, 1, -1>(f), p0 = row_sum<Q, 1, 0>(f), pp = row_sum<Q, 1, 1>(f);
    Moments m;
    const float ayp = pm.A + p0.A + pp.A, aym = mm.A + m0.A + mp.A;
    const float azp = mp.A + op.A + pp.A, azm = mm.A + om.A + pm.A;
    m.s0 = (ayp + aym) + (om.A + oo.A + op.A);
    m.jy = ayp - aym;
    m.pyy = ayp + aym;
    m.jz = azp - azm;
    m.pzz = azp + azm;
    m.pyz = (pp.A + mm.A) - (pm.A + mp.A);
    if constexpr (Q == 27) {
        const float xyp = pm.X + p0.X + pp.X, xym = mm.X + m0.X + mp.X;
        m.jx = (xyp + xym) + (om.X + oo.X + op.X);
        m.pxy = xyp - xym;
        m.pxz = (mp.X + op.X + pp.X) - (mm.X + om.X + pm.X);
        m.pxx = ((pm.B + p0.B + pp.B) + (mm.B + m0.B + mp.B)) + (om.B + oo.B + op.B);
    } else {
        m.jx = (p0.X + m0.X) + (oo.X + (op.X + om.X));
        m.pxy = p0.X - m0.X;
        m.pxz = op.X - om.X;
        m.pxx = (p0.B + m0.B) + (oo.B + (op.B + om.B));
    }
    return m;
}

// Constants of the pair emission (see collide()): per opposite pair with
// cu = c.u, cac = c.a2.c, cau = c.a2.u,
//   E = w (C0 + R45 cu^2 + K45 cac),  O = w (cu (D0 + R45o cu^2 + K135 cac) - K9 cau),
//   f'(c) = E + O, f'(-c) = E - O (O negated at a solid cell).
struct EmitConst {
    float C0, D0, R45, R45o, K45, K135, K9;
    float ux, uy, uz, vx, vy, vz;
    float axx, ayy, azz, axy2, axz2, ayz2, syz;
    float ow[4];          // w * scale per speed class, negated at a solid cell (swap of m_solids.F90:28-32)
};

// 2^8 for FP16 storage of scaled offsets, 1 for FP32
template <typename S>
__host__ __device__ constexpr float store_scale() { return sizeof(S) == 2 ? 256.0f : 1.0f; }

template <int Q, typename S, int L>
__device__ __forceinline__ void emit_pair(float (&fp)[Q], const EmitConst& k, float cu, float cac, float cau) {
    constexpr float ws = lat_w<Q>(L) * store_scale<S>();
    const float cu2 = cu * cu;
    const float E = ws * fmaf(k.K45, cac, fmaf(k.R45, cu2, k.C0));
    const float O = k.ow[lat_speed2(L)] * fmaf(-k.K9, cau, cu * fmaf(k.K135, cac, fmaf(k.R45o, cu2, k.D0)));
    fp[L] = E + O;
    fp[lat_opposite(L)] = E - O;
}

// cy*y + cz*z for cy, cz in {-1,0,1}, not both zero, without adding zeros
template <int CY, int CZ>
__device__ __forceinline__ float lin(float y, float z) {
    if constexpr (CY == 0) return CZ > 0 ? z : -z;
    else if constexpr (CZ == 0) return CY > 0 ? y : -y;
    else return (CY > 0 ? y : -y) + (CZ > 0 ? z : -z);
}

// one row (CY, CZ) != (0, 0) with CY > 0 or (CY == 0 and CZ > 0): its directions and their opposites
template <int Q, typename S, int CY, int CZ>
__device__ __forceinline__ void emit_row(float (&fp)[Q], const EmitConst& k) {
    using R = Row<Q, CY, CZ>;
    // (cy, cz) parts of c.u, c.a2.u and c.a2.c, and the cx coefficient of c.a2.c
    const float uyz = lin<CY, CZ>(k.uy, k.uz);
    const float vyz = lin<CY, CZ>(k.vy, k.vz);
    float ayz;
    if constexpr (CY != 0 && CZ != 0) ayz = (CY * CZ > 0) ? k.syz + k.ayz2 : k.syz - k.ayz2;
    else ayz = (CY != 0) ? k.ayy : k.azz;
    emit_pair<Q, S, R::l0>(fp, k, uyz, ayz, vyz);
    if constexpr (R::hasx) {
        const float bx = lin<CY, CZ>(k.axy2, k.axz2);
        const float t = k.axx + ayz;
        emit_pair<Q, S, R::lp>(fp, k, uyz + k.ux, t + bx, vyz + k.vx);
        emit_pair<Q, S, R::lm>(fp, k, uyz - k.ux, t - bx, vyz - k.vx);
    }
}

// Regularized collision of one cell from its moments (ihrr = 1).  fp receives
// the post-collision offsets times store_scale<S>(); returns tau.
template <int Q, typename S>
__device__ __forceinline__ float collide_rows(float (&fp)[Q], const Moments& m, float drho, float rho, float ux,
                                              float uy, float uz, const CollideParams& cp, float abl, bool solid) {
    const float third = 1.0f / 3.0f;
    const float rux = rho * ux, ruy = rho * uy, ruz = rho * uz;
    const float axx = m.pxx - m.s0 * third - rux * ux;
    const float ayy = m.pyy - m.s0 * third - ruy * uy;
    const float azz = m.pzz - m.s0 * third - ruz * uz;
    const float axy = m.pxy - rux * uy;
    const float axz = m.pxz - rux * uz;
    const float ayz = m.pyz - ruy * uz;
    const float tr = axx + ayy + azz;
    float tau = cp.tau0;
    if (cp.ivreman) {
        const float xx = axx * axx, yy = ayy * ayy, zz = azz * azz;
        const float xy = axy * axy, xz = axz * axz, yz = ayz * ayz;
        const float amag = fmaxf(xx + yy + zz + 2.0f * (xy + xz + yz), 1.17549435e-38f);
        const float b11 = cp.eps + xx + xy + xz;
        const float b22 = cp.eps + xy + yy + yz;
        const float b33 = cp.eps + xz + yz + zz;
        const float b12 = cp.eps + axx * axy + axy * ayy + axz * ayz;
        const float b13 = cp.eps + axx * axz + axy * ayz + axz * azz;
        const float b23 = cp.eps + axy * axz + ayy * ayz + ayz * azz;
        const float bb = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
        const float t = bb / amag;
        const float nut = (t > cp.eps) ? cp.cvre * sqrtf(t) : 0.0f;
        tau = 3.0f * (cp.kinevisc + nut + abl) + 0.5f;
    }
    const float K = 1.0f - __frcp_rn(tau);
    const bool cubic = (cp.ibgk == 3);
    const float usq = ux * ux + uy * uy + uz * uz;
    EmitConst k;
    k.R45 = 4.5f * rho;
    k.R45o = cubic ? k.R45 : 0.0f;
    k.C0 = (drho - 1.5f * rho * usq) - 1.5f * K * tr;
    k.D0 = (3.0f * rho - (cubic ? k.R45 * usq : 0.0f)) - 4.5f * K * tr;
    k.K45 = 4.5f * K;
    k.K135 = 13.5f * K;
    k.K9 = 9.0f * K;
    k.ux = ux; k.uy = uy; k.uz = uz;
    k.vx = axx * ux + axy * uy + axz * uz;
    k.vy = axy * ux + ayy * uy + ayz * uz;
    k.vz = axz * ux + ayz * uy + azz * uz;
    k.axx = axx; k.ayy = ayy; k.azz = azz;
    k.axy2 = 2.0f * axy; k.axz2 = 2.0f * axz; k.ayz2 = 2.0f * ayz;
    k.syz = ayy + azz;
    {
        const float sg = solid ? -store_scale<S>() : store_scale<S>();
        k.ow[0] = 0.0f;
        k.ow[1] = sg * lat_w<Q>(1);
        k.ow[2] = sg * lat_w<Q>(7);
        k.ow[3] = (Q == 27) ? sg * lat_w<27>(19) : 0.0f;
    }
    fp[0] = (lat_w<Q>(0) * store_scale<S>()) * k.C0;
    emit_pair<Q, S, Row<Q, 0, 0>::lp>(fp, k, ux, axx, k.vx);   // x faces
    emit_row<Q, S, 0, 1>(fp, k);
    emit_row<Q, S, 1, 0>(fp, k);
    emit_row<Q, S, 1, 1>(fp, k);
    emit_row<Q, S, 1, -1>(fp, k);
    return tau;
}

// Turbulence increment feq(rho, u+du) - feq(rho, u) added after the emission;
// at a solid cell the increments are swapped with the populations they belong to.
// Every operation rounds explicitly (the _rn intrinsics): plain a*b + c may be
// fused differently in kernels compiled with different register budgets, and
// the batched ensemble must reproduce the single-state kernels bit for bit.
__device__ __forceinline__ float cdot_rn(int cx, int cy, int cz, float x, float y, float z) {
    float r = 0.0f;
    if (cx) r = cx > 0 ? __fadd_rn(r, x) : __fsub_rn(r, x);
    if (cy) r = cy > 0 ? __fadd_rn(r, y) : __fsub_rn(r, y);
    if (cz) r = cz > 0 ? __fadd_rn(r, z) : __fsub_rn(r, z);
    return r;
}

template <int Q>
__device__ __forceinline__ void add_turbulence(float (&fp)[Q], float rho, float ux, float uy, float uz,
                                               const TurbIn& tb, bool cubic, bool solid, float scale) {
    const float usq = __fmaf_rn(ux, ux, __fmaf_rn(uy, uy, __fmul_rn(uz, uz)));
    const float dusq = __fmaf_rn(tb.dux, __fmaf_rn(2.0f, ux, tb.dux),
                                 __fmaf_rn(tb.duy, __fmaf_rn(2.0f, uy, tb.duy), __fmul_rn(tb.duz, __fmaf_rn(2.0f, uz, tb.duz))));
    const float usq2 = __fadd_rn(usq, dusq);
    const float sg = solid ? -1.0f : 1.0f;
    fp[0] = __fmaf_rn(__fmul_rn(lat_w<Q>(0) * scale, rho), __fmul_rn(-1.5f, dusq), fp[0]);
#pragma unroll
    for (int l = 1; l < Q; l += 2) {
        const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
        const float wr = __fmul_rn(lat_w<Q>(l) * scale, rho);
        const float cu = cdot_rn(cx, cy, cz, ux, uy, uz);
        const float dcu = cdot_rn(cx, cy, cz, tb.dux, tb.duy, tb.duz);
        const float cun = __fadd_rn(cu, dcu);
        // 4.5 dcu (2 cu + dcu) - 1.5 dusq
        const float e = __fmaf_rn(__fmul_rn(4.5f, dcu), __fmaf_rn(2.0f, cu, dcu), __fmul_rn(-1.5f, dusq));
        const float dE = __fmul_rn(wr, e);
        float od = __fmul_rn(3.0f, dcu);
        if (cubic) {
            // + 4.5 dcu (cun^2 + cun cu + cu^2 - usq2) - 4.5 cu dusq
            const float poly = __fsub_rn(__fmaf_rn(cun, __fadd_rn(cun, cu), __fmul_rn(cu, cu)), usq2);
            od = __fmaf_rn(__fmul_rn(4.5f, dcu), poly, od);
            od = __fmaf_rn(__fmul_rn(-4.5f, cu), dusq, od);
        }
        const float dO = __fmul_rn(__fmul_rn(sg, wr), od);
        fp[l] = __fadd_rn(fp[l], __fadd_rn(dE, dO));
        fp[l + 1] = __fadd_rn(fp[l + 1], __fsub_rn(dE, dO));
    }
}

}  // namespace lbm
