// sep_emit.cuh -- the D3Q27 post-collision populations of two cells by a
// separable transform (FP16-offset state).
//
// The regularized post-collision population of direction c (collide_rows.cuh,
// with K = 1 - 1/tau and the non-equilibrium moments a) is w_c P(c), where
//   P(c) = C0 + 4.5 K c.a.c + 4.5 rho (c.u)^2
//        + s [ -9 K c.a.u + (c.u) (D0 + 13.5 K c.a.c + 4.5 rho_c (c.u)^2) ],
// s = -1 at a solid cell (the swap of opposite directions negates the odd part)
// and rho_c = rho for the third-order equilibrium, 0 for the second.  P is a
// cubic in (cx, cy, cz) on {-1, 0, 1}^3, so with cx^3 = cx it has 17 nonzero
// coefficients in the product basis {1, c, c^2} of each axis, and the D3Q27
// weights factor by axis: w(c) = (8/27) r(cx) r(cy) r(cz), r(0) = 1,
// r(+-1) = 1/4.  All 27 values therefore follow from the coefficients by three
// one-axis passes (z, then y, then x), each turning coefficients (b0, b1, b2)
// of one axis into the values at c = 0, +1, -1:
//   v(0) = b0,  v(+-1) = (b0 + b2 +- b1) / 4,
// with the coefficients prescaled by 1/4 per nonzero index so that a pass is a
// fused multiply-add and two additions.  The transform takes 74 packed
// operations where the direction-by-direction emission of collide_rows2 takes
// about 180; the FP16 state, whose step runs short of issue slots before it
// runs short of bandwidth, is where that pays.
//
// The inflow-turbulence increment feq(rho, u + du) - feq(rho, u) of the forcing
// slice (m_inflow_turbulence_forcing.F90:41-125) is a cubic of the same form,
// so the slice cell adds its coefficients before the transform instead of
// adding 27 increments after it.
#pragma once

// included from pair_step.cuh (needs f2 helpers, CollideState2, pair_edge)

namespace lbm {

struct SepCoef {
    f2 t000;                                 // 1
    f2 t200, t020, t002, t110, t101, t011;   // cx^2, cy^2, cz^2, cx cy, cx cz, cy cz
    f2 t100, t010, t001;                     // cx, cy, cz
    f2 t210, t201, t120, t021, t102, t012;   // cx^2 cy, cx^2 cz, cx cy^2, cy^2 cz, cx cz^2, cy cz^2
    f2 t111;                                 // cx cy cz
};

// prescale of a coefficient with n nonzero indices: store scale x 8/27 / 4^n
template <typename S, int N>
__host__ __device__ constexpr float sep_beta() {
    return store_scale<S>() * (8.0f / 27.0f) / (N == 0 ? 1.0f : N == 1 ? 4.0f : N == 2 ? 16.0f : 64.0f);
}

template <typename S>
__device__ __forceinline__ SepCoef sep_coefficients(const CollideState2& c, f2 sg, bool cubic) {
    const f2 ux = c.ux, uy = c.uy, uz = c.uz, K = c.K, rho = c.rho;
    const f2 axx = c.axx, ayy = c.ayy, azz = c.azz, axy = c.axy, axz = c.axz, ayz = c.ayz;
    SepCoef t;
    const f2 qx = mul2(ux, ux), qy = mul2(uy, uy), qz = mul2(uz, uz);
    const f2 rqx = mul2(c.rux, ux), rqy = mul2(c.ruy, uy), rqz = mul2(c.ruz, uz);   // rho u_a^2
    const f2 rusq = add2(add2(rqx, rqy), rqz);
    const f2 ktr = mul2(K, c.tr);
    // even part
    t.t000 = mul2(bc2(sep_beta<S, 0>()), fma2(bc2(-1.5f), ktr, fma2(bc2(-1.5f), rusq, c.drho)));
    const f2 e1 = bc2(4.5f * sep_beta<S, 1>()), e2 = bc2(9.0f * sep_beta<S, 2>());
    t.t200 = mul2(e1, fma2(K, axx, rqx));
    t.t020 = mul2(e1, fma2(K, ayy, rqy));
    t.t002 = mul2(e1, fma2(K, azz, rqz));
    t.t110 = mul2(e2, fma2(K, axy, mul2(c.rux, uy)));
    t.t101 = mul2(e2, fma2(K, axz, mul2(c.rux, uz)));
    t.t011 = mul2(e2, fma2(K, ayz, mul2(c.ruy, uz)));
    // odd part, with the solid sign
    const f2 rc = cubic ? rho : bc2(0.0f);
    const f2 sK = mul2(sg, K), sR = mul2(sg, rc);
    // D0 = 3 rho - 4.5 rho_c u^2 - 4.5 K tr
    const f2 sD = mul2(sg, fma2(bc2(-4.5f), mul2(rc, add2(add2(qx, qy), qz)), fma2(bc2(-4.5f), ktr, mul2(bc2(3.0f), rho))));
    const f2 vx = fma2(axx, ux, fma2(axy, uy, mul2(axz, uz)));
    const f2 vy = fma2(axy, ux, fma2(ayy, uy, mul2(ayz, uz)));
    const f2 vz = fma2(axz, ux, fma2(ayz, uy, mul2(azz, uz)));
    const f2 A1 = mul2(bc2(13.5f * sep_beta<S, 1>()), sK), B1 = mul2(bc2(4.5f * sep_beta<S, 1>()), sR);
    const f2 D1 = mul2(bc2(sep_beta<S, 1>()), sD), N1 = mul2(bc2(-9.0f * sep_beta<S, 1>()), sK);
    t.t100 = fma2(N1, vx, mul2(ux, fma2(A1, axx, fma2(B1, qx, D1))));
    t.t010 = fma2(N1, vy, mul2(uy, fma2(A1, ayy, fma2(B1, qy, D1))));
    t.t001 = fma2(N1, vz, mul2(uz, fma2(A1, azz, fma2(B1, qz, D1))));
    // c_a c_b^2: 13.5 K (u_a a_bb + 2 u_b a_ab) + 13.5 rho_c u_a u_b^2 = u_a P_b + u_b Q_ab
    const f2 A2 = mul2(bc2(13.5f * sep_beta<S, 2>()), sK), B2 = mul2(bc2(13.5f * sep_beta<S, 2>()), sR);
    const f2 Px = fma2(A2, axx, mul2(B2, qx)), Py = fma2(A2, ayy, mul2(B2, qy)), Pz = fma2(A2, azz, mul2(B2, qz));
    const f2 A2t = add2(A2, A2);
    const f2 Qxy = mul2(A2t, axy), Qxz = mul2(A2t, axz), Qyz = mul2(A2t, ayz);
    t.t120 = fma2(ux, Py, mul2(uy, Qxy));
    t.t102 = fma2(ux, Pz, mul2(uz, Qxz));
    t.t210 = fma2(uy, Px, mul2(ux, Qxy));
    t.t012 = fma2(uy, Pz, mul2(uz, Qyz));
    t.t201 = fma2(uz, Px, mul2(ux, Qxz));
    t.t021 = fma2(uz, Py, mul2(uy, Qyz));
    // cx cy cz: 27 K (ux ayz + uy axz + uz axy) + 27 rho_c ux uy uz
    const f2 A3 = mul2(bc2(27.0f * sep_beta<S, 3>()), sK), B3 = mul2(bc2(27.0f * sep_beta<S, 3>()), sR);
    t.t111 = fma2(B3, mul2(mul2(ux, uy), uz), mul2(A3, fma2(ux, ayz, fma2(uy, axz, mul2(uz, axy)))));
    return t;
}

__device__ __forceinline__ void sep_add(f2& v, int comp, float d) {
    if (comp) v.y = __fadd_rn(v.y, d);
    else v.x = __fadd_rn(v.x, d);
}

// The turbulence increment feq(rho, u + du) - feq(rho, u) of one cell (component
// comp of the pair) added to the coefficients: 3 c.du + 4.5 ((c.u')^2 - (c.u)^2)
// - 1.5 (u'^2 - u^2) + 4.5 [(c.u')^3 - (c.u)^3 - (c.u') u'^2 + (c.u) u^2] (cubic),
// u' = u + du, times rho, the odd part with the solid sign (add_turbulence of
// collide_rows.cuh, coefficient by coefficient).
template <typename S>
__device__ __forceinline__ void sep_add_turbulence(SepCoef& t, int comp, float rho, float ux, float uy, float uz,
                                                   const TurbIn& tb, bool cubic, bool solid) {
    // explicit roundings throughout (see add_turbulence in collide_rows.cuh)
    const float vx = __fadd_rn(ux, tb.dux), vy = __fadd_rn(uy, tb.duy), vz = __fadd_rn(uz, tb.duz);
    const float usq = __fmaf_rn(ux, ux, __fmaf_rn(uy, uy, __fmul_rn(uz, uz)));
    const float dx = __fmul_rn(tb.dux, __fmaf_rn(2.0f, ux, tb.dux));     // u'x^2 - ux^2
    const float dy = __fmul_rn(tb.duy, __fmaf_rn(2.0f, uy, tb.duy));
    const float dz = __fmul_rn(tb.duz, __fmaf_rn(2.0f, uz, tb.duz));
    const float dusq = __fadd_rn(__fadd_rn(dx, dy), dz);
    const float vsq = __fadd_rn(usq, dusq);
    const float s = solid ? -rho : rho;
    const float c3 = cubic ? 1.0f : 0.0f;
    // difference of products p(u') - p(u), u' = u + du
    auto d2 = [](float a1, float b1, float a0, float b0) { return __fmaf_rn(a1, b1, -__fmul_rn(a0, b0)); };
    auto d3 = [](float a1, float b1, float c1, float a0, float b0, float c0) {
        return __fmaf_rn(__fmul_rn(a1, b1), c1, -__fmul_rn(__fmul_rn(a0, b0), c0));
    };
    sep_add(t.t000, comp, __fmul_rn(sep_beta<S, 0>() * -1.5f, __fmul_rn(rho, dusq)));
    const float e1 = __fmul_rn(4.5f * sep_beta<S, 1>(), rho), e2 = __fmul_rn(9.0f * sep_beta<S, 2>(), rho);
    sep_add(t.t200, comp, __fmul_rn(e1, dx));
    sep_add(t.t020, comp, __fmul_rn(e1, dy));
    sep_add(t.t002, comp, __fmul_rn(e1, dz));
    sep_add(t.t110, comp, __fmul_rn(e2, d2(vx, vy, ux, uy)));
    sep_add(t.t101, comp, __fmul_rn(e2, d2(vx, vz, ux, uz)));
    sep_add(t.t011, comp, __fmul_rn(e2, d2(vy, vz, uy, uz)));
    const float o1 = __fmul_rn(sep_beta<S, 1>(), s), k3 = __fmul_rn(4.5f, c3);
    // 3 du_a + 4.5 [(u'_a^3 - u_a^3) - (u'_a u'^2 - u_a u^2)]
    sep_add(t.t100, comp, __fmul_rn(o1, __fmaf_rn(k3, __fsub_rn(d3(vx, vx, vx, ux, ux, ux), d2(vx, vsq, ux, usq)),
                                                   __fmul_rn(3.0f, tb.dux))));
    sep_add(t.t010, comp, __fmul_rn(o1, __fmaf_rn(k3, __fsub_rn(d3(vy, vy, vy, uy, uy, uy), d2(vy, vsq, uy, usq)),
                                                   __fmul_rn(3.0f, tb.duy))));
    sep_add(t.t001, comp, __fmul_rn(o1, __fmaf_rn(k3, __fsub_rn(d3(vz, vz, vz, uz, uz, uz), d2(vz, vsq, uz, usq)),
                                                   __fmul_rn(3.0f, tb.duz))));
    const float o2 = __fmul_rn(__fmul_rn(13.5f * sep_beta<S, 2>(), s), c3);
    sep_add(t.t120, comp, __fmul_rn(o2, d3(vx, vy, vy, ux, uy, uy)));
    sep_add(t.t102, comp, __fmul_rn(o2, d3(vx, vz, vz, ux, uz, uz)));
    sep_add(t.t210, comp, __fmul_rn(o2, d3(vx, vx, vy, ux, ux, uy)));
    sep_add(t.t012, comp, __fmul_rn(o2, d3(vy, vz, vz, uy, uz, uz)));
    sep_add(t.t201, comp, __fmul_rn(o2, d3(vx, vx, vz, ux, ux, uz)));
    sep_add(t.t021, comp, __fmul_rn(o2, d3(vy, vy, vz, uy, uy, uz)));
    sep_add(t.t111, comp, __fmul_rn(__fmul_rn(__fmul_rn(27.0f * sep_beta<S, 3>(), s), c3), d3(vx, vy, vz, ux, uy, uz)));
}

// one axis: coefficients (b0, b1/4, b2/4) -> values at 0, +1, -1
struct Tri {
    f2 o, p, m;
};
__device__ __forceinline__ Tri tri3(f2 b0, f2 b1, f2 b2) {
    const f2 t = fma2(b0, bc2(0.25f), b2);
    return {b0, add2(t, b1), sub2(t, b1)};
}
__device__ __forceinline__ Tri tri2(f2 b0, f2 b1) {
    const f2 t = mul2(b0, bc2(0.25f));
    return {b0, add2(t, b1), sub2(t, b1)};
}
__device__ __forceinline__ Tri tri1(f2 b0) {
    const f2 t = mul2(b0, bc2(0.25f));
    return {b0, t, t};
}
template <int C>
__device__ __forceinline__ f2 tri_at(const Tri& t) {
    return C == 0 ? t.o : (C > 0 ? t.p : t.m);
}

// the x pass for one (cy, cz): hands the three values to sink(L, value)
template <int CY, int CZ, typename Sink>
__device__ __forceinline__ void sep_x(const Tri& h0, const Tri& h1, const Tri& h2, Sink& sink) {
    const Tri v = tri3(tri_at<CY>(h0), tri_at<CY>(h1), tri_at<CY>(h2));
    sink.template put<lat_find<27>(0, CY, CZ)>(v.o);
    sink.template put<lat_find<27>(1, CY, CZ)>(v.p);
    sink.template put<lat_find<27>(-1, CY, CZ)>(v.m);
}

// the y and x passes for one cz
template <int CZ, typename Sink>
__device__ __forceinline__ void sep_yx(const Tri& g00, const Tri& g01, const Tri& g02, const Tri& g10, const Tri& g11,
                                       const Tri& g12, const Tri& g20, const Tri& g21, Sink& sink) {
    const Tri h0 = tri3(tri_at<CZ>(g00), tri_at<CZ>(g01), tri_at<CZ>(g02));
    const Tri h1 = tri3(tri_at<CZ>(g10), tri_at<CZ>(g11), tri_at<CZ>(g12));
    const Tri h2 = tri2(tri_at<CZ>(g20), tri_at<CZ>(g21));
    sep_x<0, CZ>(h0, h1, h2, sink);
    sep_x<1, CZ>(h0, h1, h2, sink);
    sep_x<-1, CZ>(h0, h1, h2, sink);
}

// all 27 values of the pair, in the store scale, to sink.put<L>(value)
template <typename Sink>
__device__ __forceinline__ void sep_transform27(const SepCoef& t, Sink& sink) {
    const Tri g00 = tri3(t.t000, t.t001, t.t002);
    const Tri g10 = tri3(t.t100, t.t101, t.t102);
    const Tri g01 = tri3(t.t010, t.t011, t.t012);
    const Tri g20 = tri2(t.t200, t.t201);
    const Tri g02 = tri2(t.t020, t.t021);
    const Tri g11 = tri2(t.t110, t.t111);
    const Tri g21 = tri1(t.t210);
    const Tri g12 = tri1(t.t120);
    sep_yx<0>(g00, g01, g02, g10, g11, g12, g20, g21, sink);
    sep_yx<1>(g00, g01, g02, g10, g11, g12, g20, g21, sink);
    sep_yx<-1>(g00, g01, g02, g10, g11, g12, g20, g21, sink);
}

}  // namespace lbm
