// pair_step.cuh -- the steady fused step with two cells per thread on the
// packed FP32 pipes of sm_100 (fma/add/mul .f32x2).
//
// Same update as k_step_fast with the regularized collision of
// collide_rows.cuh (ihrr = 1), for the cells (i, i+1), i odd, of one row: every
// arithmetic step of the collision runs once for both cells as one f32x2
// instruction, and the memory side moves both cells at once: an aligned
// float2 / half2 load for the directions with cx = 0, two loads (FP32) or two
// words and a byte permute (FP16) for cx = +-1, one float2 / half2 store per
// direction.  The per-cell divisions, reciprocals and square roots of the
// Vreman model stay scalar.
//
// Layout facts this relies on: interior i = 1 sits at an even element of its
// row, the row pitch and the direction stride are even, so the first cell of a
// pair is 8-byte (FP32) / 4-byte (FP16) aligned; nx is even.
#pragma once

#include "state_kernels.cuh"

namespace lbm {

using f2 = float2;

__device__ __forceinline__ f2 bc2(float s) { return make_float2(s, s); }
__device__ __forceinline__ f2 add2(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 sub2(f2 a, f2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }   // exact a - b
__device__ __forceinline__ f2 mul2(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }

struct RowSum2 {
    f2 A, X, B;
};

template <int Q, int CY, int CZ>
__device__ __forceinline__ RowSum2 row_sum2(const f2 (&f)[Q]) {
    using R = Row<Q, CY, CZ>;
    RowSum2 s;
    if constexpr (R::hasx) {
        s.B = add2(f[R::lp], f[R::lm]);
        s.X = sub2(f[R::lp], f[R::lm]);
        s.A = add2(s.B, f[R::l0]);
    } else {
        s.B = bc2(0.f);
        s.X = bc2(0.f);
        s.A = f[R::l0];
    }
    return s;
}

struct Moments2 {
    f2 s0, jx, jy, jz, pxx, pyy, pzz, pxy, pxz, pyz;
};

// moments_rows() of collide_rows.cuh for two cells
template <int Q>
__device__ __forceinline__ Moments2 moments_rows2(const f2 (&f)[Q]) {
    const RowSum2 mm = row_sum2<Q, -1, -1>(f), m0 = row_sum2<Q, -1, 0>(f), mp = row_sum2<Q, -1, 1>(f);
    const RowSum2 om = row_sum2<Q, 0, -1>(f), oo = row_sum2<Q, 0, 0>(f), op = row_sum2<Q, 0, 1>(f);
    const RowSum2 pm = row_sum2<Q, 1, -1>(f), p0 = row_sum2<Q, 1, 0>(f), pp = row_sum2<Q, 1, 1>(f);
    Moments2 m;
    const f2 ayp = add2(add2(pm.A, p0.A), pp.A), aym = add2(add2(mm.A, m0.A), mp.A);
    const f2 azp = add2(add2(mp.A, op.A), pp.A), azm = add2(add2(mm.A, om.A), pm.A);
    m.s0 = add2(add2(ayp, aym), add2(add2(om.A, oo.A), op.A));
    m.jy = sub2(ayp, aym);
    m.pyy = add2(ayp, aym);
    m.jz = sub2(azp, azm);
    m.pzz = add2(azp, azm);
    m.pyz = sub2(add2(pp.A, mm.A), add2(pm.A, mp.A));
    if constexpr (Q == 27) {
        const f2 xyp = add2(add2(pm.X, p0.X), pp.X), xym = add2(add2(mm.X, m0.X), mp.X);
        m.jx = add2(add2(xyp, xym), add2(add2(om.X, oo.X), op.X));
        m.pxy = sub2(xyp, xym);
        m.pxz = sub2(add2(add2(mp.X, op.X), pp.X), add2(add2(mm.X, om.X), pm.X));
        m.pxx = add2(add2(add2(add2(pm.B, p0.B), pp.B), add2(add2(mm.B, m0.B), mp.B)), add2(add2(om.B, oo.B), op.B));
    } else {
        m.jx = add2(add2(p0.X, m0.X), add2(oo.X, add2(op.X, om.X)));
        m.pxy = sub2(p0.X, m0.X);
        m.pxz = sub2(op.X, om.X);
        m.pxx = add2(add2(p0.B, m0.B), add2(oo.B, add2(op.B, om.B)));
    }
    return m;
}

// EmitConst of collide_rows.cuh for two cells (nK9 = -K9)
struct EmitConst2 {
    f2 C0, D0, R45, R45o, K45, K135, nK9;
    f2 ux, uy, uz, vx, vy, vz;
    f2 axx, ayy, azz, axy2, axz2, ayz2, syz;
    f2 ow[4];
};

template <int Q, typename S, int L>
__device__ __forceinline__ void emit_pair2(f2 (&fp)[Q], const EmitConst2& k, f2 cu, f2 cac, f2 cau) {
    const f2 ws = bc2(lat_w<Q>(L) * store_scale<S>());
    const f2 cu2 = mul2(cu, cu);
    const f2 E = mul2(ws, fma2(k.K45, cac, fma2(k.R45, cu2, k.C0)));
    const f2 O = mul2(k.ow[lat_speed2(L)], fma2(k.nK9, cau, mul2(cu, fma2(k.K135, cac, fma2(k.R45o, cu2, k.D0)))));
    fp[L] = add2(E, O);
    fp[lat_opposite(L)] = sub2(E, O);
}

// cy*y + cz*z for the rows emitted below (leading coefficient +1)
template <int CY, int CZ>
__device__ __forceinline__ f2 lin2(f2 y, f2 z) {
    static_assert(CY > 0 || (CY == 0 && CZ > 0), "row with a positive leading coefficient");
    if constexpr (CY == 0) return z;
    else if constexpr (CZ == 0) return y;
    else if constexpr (CZ > 0) return add2(y, z);
    else return sub2(y, z);
}

template <int Q, typename S, int CY, int CZ>
__device__ __forceinline__ void emit_row2(f2 (&fp)[Q], const EmitConst2& k) {
    using R = Row<Q, CY, CZ>;
    const f2 uyz = lin2<CY, CZ>(k.uy, k.uz);
    const f2 vyz = lin2<CY, CZ>(k.vy, k.vz);
    f2 ayz;
    if constexpr (CY != 0 && CZ != 0) ayz = (CY * CZ > 0) ? add2(k.syz, k.ayz2) : sub2(k.syz, k.ayz2);
    else ayz = (CY != 0) ? k.ayy : k.azz;
    emit_pair2<Q, S, R::l0>(fp, k, uyz, ayz, vyz);
    if constexpr (R::hasx) {
        const f2 bx = lin2<CY, CZ>(k.axy2, k.axz2);
        const f2 t = add2(k.axx, ayz);
        emit_pair2<Q, S, R::lp>(fp, k, add2(uyz, k.ux), add2(t, bx), add2(vyz, k.vx));
        emit_pair2<Q, S, R::lm>(fp, k, sub2(uyz, k.ux), sub2(t, bx), sub2(vyz, k.vx));
    }
}

__device__ __forceinline__ float vreman_nut(float bb, float amag, const CollideParams& cp) {
    const float t = bb / amag;
    return (t > cp.eps) ? __fmul_rn(cp.cvre, sqrtf(t)) : 0.0f;
}

// Reciprocal and square root by the approximate PTX instructions (rcp.approx,
// sqrt.approx: one special-function instruction each, relative error a few
// units in the last FP32 place).  The FP16-offset state keeps 11 significant
// bits, so these errors vanish in its rounding, while the correctly rounded
// forms cost a dozen instructions and a branch each; the FP32 state keeps the
// correctly rounded forms.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// 1/x of both cells: correctly rounded for FP32 storage, approximate for FP16
template <typename S>
__device__ __forceinline__ f2 rcp2(f2 x) {
    if constexpr (sizeof(S) == 2) return make_float2(rcp_approx(x.x), rcp_approx(x.y));
    else return make_float2(__frcp_rn(x.x), __frcp_rn(x.y));
}
// Vreman eddy viscosity of both cells from B_beta and |alpha|^2 (see vreman_nut)
template <typename S>
__device__ __forceinline__ f2 vreman_nut2(f2 bb, f2 sq, const CollideParams& cp) {
    const float tiny = 1.17549435e-38f;
    if constexpr (sizeof(S) == 2) {
        const f2 t = mul2(bb, rcp2<S>(make_float2(fmaxf(sq.x, tiny), fmaxf(sq.y, tiny))));
        return make_float2(t.x > cp.eps ? __fmul_rn(cp.cvre, sqrt_approx(t.x)) : 0.0f,
                           t.y > cp.eps ? __fmul_rn(cp.cvre, sqrt_approx(t.y)) : 0.0f);
    } else {
        return make_float2(vreman_nut(bb.x, fmaxf(sq.x, tiny), cp), vreman_nut(bb.y, fmaxf(sq.y, tiny), cp));
    }
}

// The collision state of two cells: the non-equilibrium moments a (a2 of the
// regularized collision, Pi - I S0/3 - rho u u) and, through the Vreman eddy
// viscosity, the relaxation factor K = 1 - 1/tau.
struct CollideState2 {
    f2 rho, drho, ux, uy, uz;
    f2 rux, ruy, ruz;                 // rho u
    f2 axx, ayy, azz, axy, axz, ayz, tr;
    f2 K;
};

template <typename S>
__device__ __forceinline__ CollideState2 collide_pre2(const Moments2& m, f2 drho, f2 rho, f2 ux, f2 uy, f2 uz,
                                                      const CollideParams& cp, float abl) {
    CollideState2 c;
    c.rho = rho; c.drho = drho; c.ux = ux; c.uy = uy; c.uz = uz;
    const f2 third = bc2(1.0f / 3.0f);
    const f2 rux = mul2(rho, ux), ruy = mul2(rho, uy), ruz = mul2(rho, uz);
    c.rux = rux; c.ruy = ruy; c.ruz = ruz;
    const f2 s3 = mul2(m.s0, third);
    const f2 axx = sub2(sub2(m.pxx, s3), mul2(rux, ux));
    const f2 ayy = sub2(sub2(m.pyy, s3), mul2(ruy, uy));
    const f2 azz = sub2(sub2(m.pzz, s3), mul2(ruz, uz));
    const f2 axy = sub2(m.pxy, mul2(rux, uy));
    const f2 axz = sub2(m.pxz, mul2(rux, uz));
    const f2 ayz = sub2(m.pyz, mul2(ruy, uz));
    c.axx = axx; c.ayy = ayy; c.azz = azz; c.axy = axy; c.axz = axz; c.ayz = ayz;
    c.tr = add2(add2(axx, ayy), azz);
    f2 tau = bc2(cp.tau0);
    if (cp.ivreman) {
        const f2 xx = mul2(axx, axx), yy = mul2(ayy, ayy), zz = mul2(azz, azz);
        const f2 xy = mul2(axy, axy), xz = mul2(axz, axz), yz = mul2(ayz, ayz);
        const f2 sq = fma2(bc2(2.0f), add2(add2(xy, xz), yz), add2(add2(xx, yy), zz));
        const f2 eps = bc2(cp.eps);
        const f2 b11 = add2(add2(add2(eps, xx), xy), xz);
        const f2 b22 = add2(add2(add2(eps, xy), yy), yz);
        const f2 b33 = add2(add2(add2(eps, xz), yz), zz);
        const f2 b12 = add2(eps, fma2(axx, axy, fma2(axy, ayy, mul2(axz, ayz))));
        const f2 b13 = add2(eps, fma2(axx, axz, fma2(axy, ayz, mul2(axz, azz))));
        const f2 b23 = add2(eps, fma2(axy, axz, fma2(ayy, ayz, mul2(ayz, azz))));
        f2 bb = sub2(mul2(b11, b22), mul2(b12, b12));
        bb = add2(bb, sub2(mul2(b11, b33), mul2(b13, b13)));
        bb = add2(bb, sub2(mul2(b22, b33), mul2(b23, b23)));
        const f2 nut = vreman_nut2<S>(bb, sq, cp);
        tau = fma2(bc2(3.0f), add2(bc2(cp.kinevisc + abl), nut), bc2(0.5f));
    }
    c.K = sub2(bc2(1.0f), rcp2<S>(tau));
    return c;
}

// collide_rows() for two cells: fp receives the post-collision offsets times
// store_scale<S>().  solid.x / solid.y flag the two cells.
template <int Q, typename S>
__device__ __forceinline__ void collide_rows2(f2 (&fp)[Q], const Moments2& m, f2 drho, f2 rho, f2 ux, f2 uy, f2 uz,
                                              const CollideParams& cp, float abl, bool solid0, bool solid1) {
    const CollideState2 c = collide_pre2<S>(m, drho, rho, ux, uy, uz, cp, abl);
    const f2 axx = c.axx, ayy = c.ayy, azz = c.azz, axy = c.axy, axz = c.axz, ayz = c.ayz, tr = c.tr, K = c.K;
    const bool cubic = (cp.ibgk == 3);
    const f2 usq = fma2(ux, ux, fma2(uy, uy, mul2(uz, uz)));
    EmitConst2 k;
    k.R45 = mul2(bc2(4.5f), rho);
    k.R45o = cubic ? k.R45 : bc2(0.0f);
    const f2 ktr = mul2(K, tr);
    k.C0 = sub2(sub2(drho, mul2(bc2(1.5f), mul2(rho, usq))), mul2(bc2(1.5f), ktr));
    k.D0 = sub2(sub2(mul2(bc2(3.0f), rho), cubic ? mul2(k.R45, usq) : bc2(0.0f)), mul2(bc2(4.5f), ktr));
    k.K45 = mul2(bc2(4.5f), K);
    k.K135 = mul2(bc2(13.5f), K);
    k.nK9 = mul2(bc2(-9.0f), K);
    k.ux = ux; k.uy = uy; k.uz = uz;
    k.vx = fma2(axx, ux, fma2(axy, uy, mul2(axz, uz)));
    k.vy = fma2(axy, ux, fma2(ayy, uy, mul2(ayz, uz)));
    k.vz = fma2(axz, ux, fma2(ayz, uy, mul2(azz, uz)));
    k.axx = axx; k.ayy = ayy; k.azz = azz;
    const f2 two = bc2(2.0f);
    k.axy2 = mul2(two, axy); k.axz2 = mul2(two, axz); k.ayz2 = mul2(two, ayz);
    k.syz = add2(ayy, azz);
    {
        const float s = store_scale<S>();
        const f2 sg = make_float2(solid0 ? -s : s, solid1 ? -s : s);
        k.ow[0] = bc2(0.0f);
        k.ow[1] = mul2(sg, bc2(lat_w<Q>(1)));
        k.ow[2] = mul2(sg, bc2(lat_w<Q>(7)));
        k.ow[3] = (Q == 27) ? mul2(sg, bc2(lat_w<27>(19))) : bc2(0.0f);
    }
    fp[0] = mul2(bc2(lat_w<Q>(0) * store_scale<S>()), k.C0);
    emit_pair2<Q, S, Row<Q, 0, 0>::lp>(fp, k, ux, axx, k.vx);
    emit_row2<Q, S, 0, 1>(fp, k);
    emit_row2<Q, S, 1, 0>(fp, k);
    emit_row2<Q, S, 1, 1>(fp, k);
    emit_row2<Q, S, 1, -1>(fp, k);
}

// Pull loads of the pair (i, i+1): direction L reads the pair at base + poff[L]
// (first element odd when cx != 0).
template <int Q, typename S, int L>
struct PairLoad {
    static __device__ __forceinline__ void run(f2 (&fp)[Q], const S* p0, const S* pyp, const S* pym, const StepArgs& a) {
        const S* b = reinterpret_cast<const S*>(reinterpret_cast<const char*>(lat_cy(L) > 0 ? pyp : (lat_cy(L) < 0 ? pym : p0)) + a.poffb[L]);
        if constexpr (sizeof(S) == 4) {
            if constexpr (lat_cx(L) == 0) fp[L] = __ldg(reinterpret_cast<const float2*>(b));
            else fp[L] = make_float2(__ldg(reinterpret_cast<const float*>(b)), __ldg(reinterpret_cast<const float*>(b) + 1));
        } else {
            unsigned int w;
            if constexpr (lat_cx(L) == 0) {
                w = __ldg(reinterpret_cast<const unsigned int*>(b));
            } else {
                const unsigned int w0 = __ldg(reinterpret_cast<const unsigned int*>(b - 1));
                const unsigned int w1 = __ldg(reinterpret_cast<const unsigned int*>(b + 1));
                w = __byte_perm(w0, w1, 0x5432);   // high half of w0, low half of w1
            }
            fp[L] = __half22float2(*reinterpret_cast<const __half2*>(&w));   // 2^8-scaled
        }
        PairLoad<Q, S, L + 1>::run(fp, p0, pyp, pym, a);
    }
};
template <int Q, typename S>
struct PairLoad<Q, S, Q> {
    static __device__ __forceinline__ void run(f2 (&)[Q], const S*, const S*, const S*, const StepArgs&) {}
};

__device__ __forceinline__ float comp(f2 v, int c) { return c ? v.y : v.x; }
}  // namespace lbm

#include "sep_emit.cuh"

namespace lbm {
// sep_transform27's values into the pair's population array
template <int Q>
struct SepArraySink {
    f2 (&fp)[Q];
    template <int L>
    __device__ __forceinline__ void put(f2 v) { fp[L] = v; }
};

// Everything between the loads and the stores of one pair: moments, collision,
// turbulence slice and external forcing, with the solid swap folded in.  On
// return fp holds the post-collision offsets (times store_scale<S>()).  (Variants
// that moved the turbulence slice out of the step kernel -- a one-cell post-pass,
// or a captured FP32 copy finished by a second kernel -- measured slower on B200.)
template <int Q, typename S, bool FORCE = false>
__device__ __forceinline__ void pair_collide(f2 (&fp)[Q], const StepArgs& a, int i, int j, int k) {
    Moments2 m = moments_rows2<Q>(fp);
    if constexpr (sizeof(S) == 2) {
        const f2 is = bc2(1.0f / store_scale<S>());
        m.s0 = mul2(m.s0, is); m.jx = mul2(m.jx, is); m.jy = mul2(m.jy, is); m.jz = mul2(m.jz, is);
        m.pxx = mul2(m.pxx, is); m.pyy = mul2(m.pyy, is); m.pzz = mul2(m.pzz, is);
        m.pxy = mul2(m.pxy, is); m.pxz = mul2(m.pxz, is); m.pyz = mul2(m.pyz, is);
    }
    const f2 drho = m.s0;
    const f2 rho = add2(bc2(1.0f), m.s0);
    const f2 inv = rcp2<S>(rho);
    const f2 ux = mul2(m.jx, inv), uy = mul2(m.jy, inv), uz = mul2(m.jz, inv);
    flag_bad_density2(a.status, rho, add2(add2(rho, ux), add2(uy, uz)));
    bool solid0 = false, solid1 = false;
    if (a.solid) {
        const unsigned short s2 =
            *reinterpret_cast<const unsigned short*>(a.solid + ((long long)(k - 1) * a.g.ny + (j - 1)) * a.g.nx + (i - 1));
        solid0 = (s2 & 0xffu) != 0;
        solid1 = (s2 >> 8) != 0;
    }
    const float abl = a.abl ? a.abl[k - 1] : 0.0f;
#ifndef LBM_NO_SEP
    if constexpr (Q == 27 && sizeof(S) == 2) {
        // FP16-offset D3Q27: the separable transform of sep_emit.cuh, the turbulence
        // increment folded into its coefficients
        const CollideState2 c = collide_pre2<S>(m, drho, rho, ux, uy, uz, a.cp, abl);
        const bool cubic = a.cp.ibgk == 3;
        SepCoef t = sep_coefficients<S>(c, make_float2(solid0 ? -1.0f : 1.0f, solid1 ? -1.0f : 1.0f), cubic);
        if (a.uu != nullptr && (i == a.iturb || i + 1 == a.iturb)) {
            const int cc = a.iturb - i;
            const TurbIn tb = turb_at(a, a.iturb, j, k);
            sep_add_turbulence<S>(t, cc, comp(rho, cc), comp(ux, cc), comp(uy, cc), comp(uz, cc), tb, cubic,
                                  cc ? solid1 : solid0);
        }
        SepArraySink<Q> sink{fp};
        sep_transform27(t, sink);
    } else
#endif
    {
    collide_rows2<Q, S>(fp, m, drho, rho, ux, uy, uz, a.cp, abl, solid0, solid1);
    if (a.uu != nullptr && (i == a.iturb || i + 1 == a.iturb)) {
        const int c = a.iturb - i;
        float t[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) t[l] = comp(fp[l], c);
        const TurbIn tb = turb_at(a, a.iturb, j, k);
        add_turbulence<Q>(t, comp(rho, c), comp(ux, c), comp(uy, c), comp(uz, c), tb, a.cp.ibgk == 3, c ? solid1 : solid0,
                          store_scale<S>());
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            if (c) fp[l].y = t[l];
            else fp[l].x = t[l];
        }
    }
    }
    if constexpr (FORCE) {
        // forcings_apply (m_forcings_apply_kernel.F90:47-213): f += feq2(rho, u - F/rho) - feq2(rho, u)
        // with the pre-collision rho, u, applied before the solid swap (its odd part flips at solid cells)
        const long long c0 = (long long)i + (long long)(a.g.nx + 2) * ((long long)j + (long long)(a.g.ny + 2) * k);
        const float* F = a.force + 3 * c0;
        const bool ok0 = rho.x > 0.0f, ok1 = rho.y > 0.0f;
        const f2 dux = make_float2(ok0 ? -__ldg(F) / rho.x : 0.0f, ok1 ? -__ldg(F + 3) / rho.y : 0.0f);
        const f2 duy = make_float2(ok0 ? -__ldg(F + 1) / rho.x : 0.0f, ok1 ? -__ldg(F + 4) / rho.y : 0.0f);
        const f2 duz = make_float2(ok0 ? -__ldg(F + 2) / rho.x : 0.0f, ok1 ? -__ldg(F + 5) / rho.y : 0.0f);
        const f2 two = bc2(2.0f);
        const f2 dusq = fma2(dux, fma2(two, ux, dux), fma2(duy, fma2(two, uy, duy), mul2(duz, fma2(two, uz, duz))));
        const float sc = store_scale<S>();
        const f2 wr = mul2(bc2(sc), rho);
        const f2 sg = make_float2(solid0 ? -1.0f : 1.0f, solid1 ? -1.0f : 1.0f);
        const f2 m15 = mul2(bc2(-1.5f), dusq);
        fp[0] = fma2(mul2(bc2(lat_w<Q>(0)), wr), m15, fp[0]);
#pragma unroll
        for (int l = 1; l < Q; l += 2) {
            const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
            f2 cu = bc2(0.f), dcu = bc2(0.f);
            if (cx) { cu = cx > 0 ? add2(cu, ux) : sub2(cu, ux); dcu = cx > 0 ? add2(dcu, dux) : sub2(dcu, dux); }
            if (cy) { cu = cy > 0 ? add2(cu, uy) : sub2(cu, uy); dcu = cy > 0 ? add2(dcu, duy) : sub2(dcu, duy); }
            if (cz) { cu = cz > 0 ? add2(cu, uz) : sub2(cu, uz); dcu = cz > 0 ? add2(dcu, duz) : sub2(dcu, duz); }
            const f2 wl = mul2(bc2(lat_w<Q>(l)), wr);
            const f2 dE = mul2(wl, fma2(mul2(bc2(4.5f), dcu), fma2(two, cu, dcu), m15));
            const f2 dO = mul2(mul2(sg, wl), mul2(bc2(3.0f), dcu));
            fp[l] = add2(fp[l], add2(dE, dO));
            fp[l + 1] = add2(fp[l + 1], sub2(dE, dO));
        }
    }
}

// The edge copy of the folded boundaries: the post-collision populations of the
// pair holding i = 1 or i = nx, into the compact edge array.
template <int Q, typename S>
__device__ __forceinline__ void pair_edge(const f2 (&fp)[Q], const StepArgs& a, int i, int j, int k) {
    if (i == 1 || i + 1 == a.g.nx) {
        // the boundary kernel builds the inflow/outflow ghosts from these, read coalesced
        const long long nyz = (long long)a.g.ny * a.g.nz;
        const int c = (i == 1) ? 0 : 1;
        S* e = (S*)a.edge + (long long)c * Q * nyz + (long long)(k - 1) * a.g.ny + (j - 1);
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            if constexpr (sizeof(S) == 2) e[l * nyz] = __float2half_rn(comp(fp[l], c));   // already 2^8-scaled
            else e[l * nyz] = comp(fp[l], c);
        }
    }
}

// Everything after the loads of one pair: pair_collide, the stores and the edge
// copy of the folded boundaries (FOLD).
template <int Q, typename S, bool FOLD, bool FORCE = false>
__device__ __forceinline__ void pair_update(f2 (&fp)[Q], S* __restrict__ dst, const StepArgs& a, long long o, int i,
                                            int j, int k) {
    pair_collide<Q, S, FORCE>(fp, a, i, j, k);
    S* q = dst + o;
    if constexpr (sizeof(S) == 2) {
        // the edge copy reuses the stored half2 values (no second conversion)
        __half2 h[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            h[l] = __floats2half2_rn(fp[l].x, fp[l].y);
            *reinterpret_cast<__half2*>(reinterpret_cast<char*>(q) + a.soffb[l]) = h[l];
        }
        if (FOLD && (i == 1 || i + 1 == a.g.nx)) {
            const long long nyz = (long long)a.g.ny * a.g.nz;
            const int c = (i == 1) ? 0 : 1;
            __half* e = (__half*)a.edge + (long long)c * Q * nyz + (long long)(k - 1) * a.g.ny + (j - 1);
#pragma unroll
            for (int l = 0; l < Q; ++l) e[l * nyz] = c ? __high2half(h[l]) : __low2half(h[l]);
        }
    } else {
#pragma unroll
        for (int l = 0; l < Q; ++l) *reinterpret_cast<float2*>(reinterpret_cast<char*>(q) + a.soffb[l]) = fp[l];
        if (FOLD) pair_edge<Q, S>(fp, a, i, j, k);
    }
}

// One pair (i, i+1), i odd, of row (j, k): pull, collide, store.  WRAP: periodic
// j read through rows ny and 1; FOLD: the folded boundaries follow (edge copy).
// A j-slab tile in the folded configuration pulls its stored halo planes
// (WRAP false) and keeps the folded boundaries (FOLD true).
template <int Q, typename S, bool WRAP, bool FORCE = false, bool FOLD = WRAP>
__device__ __forceinline__ void pair_cell(const S* __restrict__ src, S* __restrict__ dst, const StepArgs& a, int i, int j,
                                          int k) {
    const long long o = a.g.off(i, j, k);
    f2 fp[Q];
    {
        const S* p0 = src + o;
        const long long wrapd = (long long)a.g.ny * a.g.pitch;
        const S* pyp = (WRAP && j == 1) ? p0 + wrapd : p0;
        const S* pym = (WRAP && j == a.g.ny) ? p0 - wrapd : p0;
        PairLoad<Q, S, 0>::run(fp, p0, pyp, pym, a);
    }
    pair_update<Q, S, FOLD, FORCE>(fp, dst, a, o, i, j, k);
}

#ifndef LBM_PAIR_MIN_BLOCKS
#define LBM_PAIR_MIN_BLOCKS 5
#endif
// FP16-offset state: lower register caps (more resident warps) without spills;
// measured best at 512x256x256: 64 registers for D3Q27 (blocks of 256 threads,
// 4 per SM, where a row's pairs fill them; else blocks of 128, 8 per SM), and
// blocks of 128, 7 per SM, for D3Q19
#ifndef LBM_PAIR_MIN_BLOCKS16_27
#define LBM_PAIR_MIN_BLOCKS16_27 8
#endif
#ifndef LBM_PAIR_MIN_BLOCKS16_19
#define LBM_PAIR_MIN_BLOCKS16_19 7
#endif
// the wide block of 256 threads: FP16 D3Q27 only
template <int Q, typename S>
__host__ __device__ constexpr bool pair_wide_ok() { return sizeof(S) == 2 && Q == 27; }
// minimum resident blocks per SM for T threads per block (the register cap)
template <int Q, typename S, int T>
__host__ __device__ constexpr int pair_min_blocks() {
    return sizeof(S) == 2 ? (Q == 27 ? LBM_PAIR_MIN_BLOCKS16_27 * 128 / T : LBM_PAIR_MIN_BLOCKS16_19) : LBM_PAIR_MIN_BLOCKS;
}
// Grid: x covers nx/2 pairs in blocks of T threads, y = j, z = k.  Needs
// ihrr = 1 and nx even; offsets are 64-bit, so any state size.
template <int Q, typename S, bool WRAP, bool FORCE = false, bool FOLD = WRAP, int T = 128>
__global__ void __launch_bounds__(T, pair_min_blocks<Q, S, T>()) k_step_pair(const S* __restrict__ src, S* __restrict__ dst,
                                                                             StepArgs a) {
    pdl_enter();
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + 1;
    if (i > a.g.nx) return;
    pair_cell<Q, S, WRAP, FORCE, FOLD>(src, dst, a, i, blockIdx.y + 1, blockIdx.z + 1);
}

}  // namespace lbm
