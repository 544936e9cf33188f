// adjoint.cuh -- reverse-mode (vector-Jacobian) kernels of the per-call path,
// in the reference layout f(nl,0:nx+1,0:ny+1,0:nz+1).
//
// Each kernel takes the adjoint of a forward kernel's outputs and returns the
// adjoint of its inputs, at the forward inputs it is given (the forward values
// are recomputed where needed, never stored):
//   postcoll   (m_postcoll_kernel.F90:70-245, regularized, optional Vreman)
//   macrovars  (m_macrovars_kernel.F90:35-49)
//   drift      (m_drift_kernel.F90:37-42): the transpose of the pull is a push
// The adjoint of solids (a swap of opposite directions) is solids itself, and
// the adjoint of boundarycond runs the boundary kernels of boundary.cuh in
// reverse order with the AdjAcc accessor below.  Derivatives are exact for the
// arithmetic of the forward kernels (collide.cuh), taken by hand.
#pragma once

#include "collide.cuh"
#include "ref_kernels.cuh"

namespace lbm {

// Reverse of one regularized collision (ihrr = 1, no turbulence slice, no solid
// flag: postcoll has none).  fp: the cell's pre-collision offsets f - w;
// gh: adjoint of the post-collision populations.  fh receives the adjoint of
// the pre-collision populations; rh, uxh, uyh, uzh are incremented by the
// adjoint of postcoll's rho, u, v, w inputs.
// The reverse of the collision up to the adjoint of its second moments (a_ij,
// with the trace and the macroscopic inputs): everything collide_adj does except
// emitting the per-direction adjoint.  m: moments of the pre-collision offsets.
struct CollideAdjOut {
    float s0h, axxh, ayyh, azzh, axyh, axzh, ayzh;
};
template <int Q>
__device__ __forceinline__ CollideAdjOut collide_adj_moments(const Moments& m, const float (&gh)[Q], float rho, float ux,
                                                             float uy, float uz, const CollideParams& cp, float abl,
                                                             float tau_in, float& rh, float& uxh, float& uyh,
                                                             float& uzh) {
    // ---- forward values (as collide()) ----
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
    float amag0 = 0.f, amag = 0.f, b11 = 0.f, b22 = 0.f, b33 = 0.f, b12 = 0.f, b13 = 0.f, b23 = 0.f, bb = 0.f, t = 0.f;
    float iamag = 0.f, st = 0.f;   // 1 / amag, sqrt(t)
    if (cp.ivreman) {
        amag0 = axx * axx + ayy * ayy + azz * azz + 2.0f * (axy * axy + axz * axz + ayz * ayz);
        amag = fmaxf(amag0, 1.17549435e-38f);
        b11 = cp.eps + axx * axx + axy * axy + axz * axz;
        b22 = cp.eps + axy * axy + ayy * ayy + ayz * ayz;
        b33 = cp.eps + axz * axz + ayz * ayz + azz * azz;
        b12 = cp.eps + axx * axy + axy * ayy + axz * ayz;
        b13 = cp.eps + axx * axz + axy * ayz + axz * azz;
        b23 = cp.eps + axy * axz + ayy * ayz + ayz * azz;
        bb = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
        iamag = 1.0f / amag;
        t = bb * iamag;
        st = sqrtf(t);
        const float nut = (t > cp.eps) ? cp.cvre * st : 0.0f;
        tau = 3.0f * (cp.kinevisc + nut + abl) + 0.5f;
    }
    const float itau = 1.0f / tau;
    const float K = 1.0f - itau;
    const bool cubic = (cp.ibgk == 3);
    const float usq = ux * ux + uy * uy + uz * uz;
    const float R45 = 4.5f * rho;
    const float R45o = cubic ? R45 : 0.0f;
    const float B0 = 3.0f * rho - (cubic ? R45 * usq : 0.0f);
    const float D0 = B0 - 4.5f * K * tr;
    const float K45 = 4.5f * K, K135 = 13.5f * K, K9 = 9.0f * K;
    const float vx = axx * ux + axy * uy + axz * uz;
    const float vy = axy * ux + ayy * uy + ayz * uz;
    const float vz = axz * ux + ayz * uy + azz * uz;

    // ---- reverse (C0 = A0 - 1.5 K tr with A0 = (rho - 1) - 1.5 rho |u|^2 enter only through their adjoints) ----
    // Emission per opposite pair (l, l+1): f(l) = E + O, f(l+1) = E - O with
    //   E / w = C0 + R45 cu^2 + K45 cac,  O / w = cu (D0 + R45o cu^2 + K135 cac) - K9 cau
    // (cu = c.u, cac = c.a.c, cau = c.a.u).  Over the pairs, sum Eh phi(c) =
    // sum_l g_l phi(c_l) for even phi and sum Oh psi(c) = sum_l g_l psi(c_l) for
    // odd psi, g_l = w_l gh_l, so every adjoint sum of the emission is a
    // contraction of the moments Gi = sum g c_i, Gij = sum g c_i c_j and
    // Gijk = sum g c_i c_j c_k (Giii = Gi since c_i^3 = c_i on these lattices).
    float C0h = lat_w<Q>(0) * gh[0];
    float Gx = 0.f, Gy = 0.f, Gz = 0.f;
    float Gxx = 0.f, Gyy = 0.f, Gzz = 0.f, Gxy = 0.f, Gxz = 0.f, Gyz = 0.f;
    float Gxxy = 0.f, Gxxz = 0.f, Gxyy = 0.f, Gyyz = 0.f, Gxzz = 0.f, Gyzz = 0.f, Gxyz = 0.f;
#pragma unroll
    for (int l = 1; l < Q; l += 2) {
        const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
        const float w = lat_w<Q>(l);
        const float Eh = w * (gh[l] + gh[l + 1]);
        const float Oh = w * (gh[l] - gh[l + 1]);
        C0h += Eh;
        macc(Gx, cx, Oh);
        macc(Gy, cy, Oh);
        macc(Gz, cz, Oh);
        macc(Gxx, cx * cx, Eh);
        macc(Gyy, cy * cy, Eh);
        macc(Gzz, cz * cz, Eh);
        macc(Gxy, cx * cy, Eh);
        macc(Gxz, cx * cz, Eh);
        macc(Gyz, cy * cz, Eh);
        macc(Gxxy, cx * cx * cy, Oh);
        macc(Gxxz, cx * cx * cz, Oh);
        macc(Gxyy, cx * cy * cy, Oh);
        macc(Gyyz, cy * cy * cz, Oh);
        macc(Gxzz, cx * cz * cz, Oh);
        macc(Gyzz, cy * cz * cz, Oh);
        macc(Gxyz, cx * cy * cz, Oh);
    }
    // Gu_i = Gij u_j; Tu_ij = Gijk u_k; Tuu_i = Tu_ij u_j; Ta_i = Gijk a_jk
    const float Gux = Gxx * ux + Gxy * uy + Gxz * uz;
    const float Guy = Gxy * ux + Gyy * uy + Gyz * uz;
    const float Guz = Gxz * ux + Gyz * uy + Gzz * uz;
    const float Tuxx = Gx * ux + Gxxy * uy + Gxxz * uz;
    const float Tuyy = Gxyy * ux + Gy * uy + Gyyz * uz;
    const float Tuzz = Gxzz * ux + Gyzz * uy + Gz * uz;
    const float Tuxy = Gxxy * ux + Gxyy * uy + Gxyz * uz;
    const float Tuxz = Gxxz * ux + Gxyz * uy + Gxzz * uz;
    const float Tuyz = Gxyz * ux + Gyyz * uy + Gyzz * uz;
    const float Tuux = Tuxx * ux + Tuxy * uy + Tuxz * uz;
    const float Tuuy = Tuxy * ux + Tuyy * uy + Tuyz * uz;
    const float Tuuz = Tuxz * ux + Tuyz * uy + Tuzz * uz;
    const float Tax = Gx * axx + Gxyy * ayy + Gxzz * azz + 2.0f * (Gxxy * axy + Gxxz * axz + Gxyz * ayz);
    const float Tay = Gxxy * axx + Gy * ayy + Gyzz * azz + 2.0f * (Gxyy * axy + Gxyz * axz + Gyyz * ayz);
    const float Taz = Gxxz * axx + Gyyz * ayy + Gz * azz + 2.0f * (Gxyz * axy + Gxzz * axz + Gyzz * ayz);
    // sum Eh cu^2, sum Eh cac, sum Oh cu, sum Oh cu^3, sum Oh cu cac, -sum Oh cau
    float R45h = Gux * ux + Guy * uy + Guz * uz;
    const float K45h = Gxx * axx + Gyy * ayy + Gzz * azz + 2.0f * (Gxy * axy + Gxz * axz + Gyz * ayz);
    const float D0h = Gx * ux + Gy * uy + Gz * uz;
    const float R45oh = Tuux * ux + Tuuy * uy + Tuuz * uz;
    const float K135h = Tuxx * axx + Tuyy * ayy + Tuzz * azz + 2.0f * (Tuxy * axy + Tuxz * axz + Tuyz * ayz);
    const float K9h = -(Gx * vx + Gy * vy + Gz * vz);
    // cu^h = 2 R45 Eh cu + Oh (D0 + 3 R45o cu^2 + K135 cac), summed with c
    uxh += 2.0f * R45 * Gux + D0 * Gx + 3.0f * R45o * Tuux + K135 * Tax;
    uyh += 2.0f * R45 * Guy + D0 * Gy + 3.0f * R45o * Tuuy + K135 * Tay;
    uzh += 2.0f * R45 * Guz + D0 * Gz + 3.0f * R45o * Tuuz + K135 * Taz;
    // cac^h = K45 Eh + K135 Oh cu, summed with c c (off-diagonal entries twice)
    float axxh = K45 * Gxx + K135 * Tuxx;
    float ayyh = K45 * Gyy + K135 * Tuyy;
    float azzh = K45 * Gzz + K135 * Tuzz;
    float axyh = 2.0f * (K45 * Gxy + K135 * Tuxy);
    float axzh = 2.0f * (K45 * Gxz + K135 * Tuxz);
    float ayzh = 2.0f * (K45 * Gyz + K135 * Tuyz);
    // cau^h = -K9 Oh, summed with c
    const float vxh = -K9 * Gx, vyh = -K9 * Gy, vzh = -K9 * Gz;
    // v = a u
    axxh += vxh * ux;
    ayyh += vyh * uy;
    azzh += vzh * uz;
    axyh += vxh * uy + vyh * ux;
    axzh += vxh * uz + vzh * ux;
    ayzh += vyh * uz + vzh * uy;
    uxh += vxh * axx + vyh * axy + vzh * axz;
    uyh += vxh * axy + vyh * ayy + vzh * ayz;
    uzh += vxh * axz + vyh * ayz + vzh * azz;
    // K45, K135, K9; C0 = A0 - 1.5 K tr; D0 = B0 - 4.5 K tr
    float Kh = 4.5f * K45h + 13.5f * K135h + 9.0f * K9h - 1.5f * tr * C0h - 4.5f * tr * D0h;
    const float trh = -1.5f * K * C0h - 4.5f * K * D0h;
    const float A0h = C0h, B0h = D0h;
    if (cubic) R45h += R45oh;
    float usqh = 0.f;
    rh += 3.0f * B0h;
    if (cubic) {
        R45h -= usq * B0h;
        usqh -= R45 * B0h;
    }
    rh += A0h * (1.0f - 1.5f * usq);
    usqh -= 1.5f * rho * A0h;
    rh += 4.5f * R45h;
    uxh += 2.0f * ux * usqh;
    uyh += 2.0f * uy * usqh;
    uzh += 2.0f * uz * usqh;
    axxh += trh;
    ayyh += trh;
    azzh += trh;
    // K = 1 - 1/tau, tau = 3 (nu + nut + abl) + 1/2, nut = cvre sqrt(bb / amag) where bb / amag > eps
    if (cp.ivreman && t > cp.eps) {
        // dK/dtau = 1/tau^2, dtau/dnut = 3, dnut/dt = cvre / (2 sqrt t), t = bb / amag
        const float th = 1.5f * Kh * itau * itau * cp.cvre / st;
        const float bbh = th * iamag;
        const float amagh = (amag0 >= 1.17549435e-38f) ? -bbh * t : 0.0f;
        const float b11h = bbh * (b22 + b33), b22h = bbh * (b11 + b33), b33h = bbh * (b11 + b22);
        const float b12h = -2.0f * b12 * bbh, b13h = -2.0f * b13 * bbh, b23h = -2.0f * b23 * bbh;
        axxh += 2.0f * axx * b11h + axy * b12h + axz * b13h + 2.0f * axx * amagh;
        ayyh += 2.0f * ayy * b22h + axy * b12h + ayz * b23h + 2.0f * ayy * amagh;
        azzh += 2.0f * azz * b33h + axz * b13h + ayz * b23h + 2.0f * azz * amagh;
        axyh += 2.0f * axy * (b11h + b22h) + (axx + ayy) * b12h + ayz * b13h + axz * b23h + 4.0f * axy * amagh;
        axzh += 2.0f * axz * (b11h + b33h) + ayz * b12h + (axx + azz) * b13h + axy * b23h + 4.0f * axz * amagh;
        ayzh += 2.0f * ayz * (b22h + b33h) + axz * b12h + axy * b13h + (ayy + azz) * b23h + 4.0f * ayz * amagh;
    }
    // a_ij = p_ij - s0/3 delta_ij - rho u_i u_j
    const float s0h = -(axxh + ayyh + azzh) * third;
    rh -= axxh * ux * ux + ayyh * uy * uy + azzh * uz * uz + axyh * ux * uy + axzh * ux * uz + ayzh * uy * uz;
    uxh -= rho * (2.0f * ux * axxh + uy * axyh + uz * axzh);
    uyh -= rho * (2.0f * uy * ayyh + ux * axyh + uz * ayzh);
    uzh -= rho * (2.0f * uz * azzh + ux * axzh + uy * ayzh);
    return CollideAdjOut{s0h, axxh, ayyh, azzh, axyh, axzh, ayzh};
}

template <int Q>
__device__ __forceinline__ void collide_adj(const float (&fp)[Q], const float (&gh)[Q], float rho, float ux, float uy,
                                            float uz, const CollideParams& cp, float abl, float tau_in, float (&fh)[Q],
                                            float& rh, float& uxh, float& uyh, float& uzh) {
    const CollideAdjOut o = collide_adj_moments<Q>(moments<Q>(fp), gh, rho, ux, uy, uz, cp, abl, tau_in, rh, uxh, uyh, uzh);
    // moments are linear in f
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
        float v = o.s0h;
        macc(v, cx * cx, o.axxh);
        macc(v, cy * cy, o.ayyh);
        macc(v, cz * cz, o.azzh);
        macc(v, cx * cy, o.axyh);
        macc(v, cx * cz, o.axzh);
        macc(v, cy * cz, o.ayzh);
        fh[l] = v;
    }
}

// postcoll adjoint over interior cells: fh holds the adjoint of postcoll's output
// f on entry and the adjoint of its input f on exit (ghost cells untouched);
// rhoh, uh, vh, wh are incremented.  f, rho, u, v, w, tau, abl: postcoll's inputs.
// blank (may be null): the adjoint of a solids call that followed postcoll is
// applied first (a swap of opposite directions at blanked cells).
template <int Q>
__global__ void __launch_bounds__(128) k_ref_postcoll_adj(float* fh, const float* f, const float* rho, const float* u,
                                                          const float* v, const float* w, const float* tau,
                                                          const float* abl, float* rhoh, float* uh, float* vh,
                                                          float* wh, const int32_t* blank, RefGrid g, CollideParams cp) {
    __shared__ float sf[128 * Q];
    __shared__ float sg[128 * Q];
    const int i0 = blockIdx.x * 128 + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
    const int n = min(128, g.nx + 1 - i0);
    const int t = threadIdx.x;
    if (n <= 0) return;
    tile_load<Q>(sf, f, g.cell(i0, j, k), n);
    tile_load<Q>(sg, fh, g.cell(i0, j, k), n);
    __syncthreads();
    if (t < n) {
        const long long c = g.cell(i0 + t, j, k);
        float fp[Q], gh[Q], out[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            fp[l] = sf[t * Q + l] - lat_w<Q>(l);
            gh[l] = sg[t * Q + l];
        }
        if (blank && blank[c] != 0) {
#pragma unroll
            for (int l = 1; l + 1 < Q; l += 2) {
                const float x = gh[l];
                gh[l] = gh[l + 1];
                gh[l + 1] = x;
            }
        }
        float rr = 0.f, ux = 0.f, uy = 0.f, uz = 0.f;
        collide_adj<Q>(fp, gh, rho[c], u[c], v[c], w[c], cp, abl ? abl[k - 1] : 0.0f, tau[c], out, rr, ux, uy, uz);
        rhoh[c] += rr;
        uh[c] += ux;
        vh[c] += uy;
        wh[c] += uz;
#pragma unroll
        for (int l = 0; l < Q; ++l) sg[t * Q + l] = out[l];
    }
    __syncthreads();
    tile_store<Q>(sg, fh, g.cell(i0, j, k), n);
}

// macrovars adjoint over the ghost-inclusive grid: fh += d(rho, u, v, w)/df^T (rhoh, uh, vh, wh)
// with rho = sum f, u = (sum c f) / rho at the forward input f.
template <int Q>
__global__ void __launch_bounds__(128) k_ref_macrovars_adj(float* fh, const float* rhoh, const float* uh,
                                                           const float* vh, const float* wh, const float* f,
                                                           RefGrid g) {
    __shared__ float sf[128 * Q];
    __shared__ float sg[128 * Q];
    const int i0 = blockIdx.x * 128, j = blockIdx.y, k = blockIdx.z;
    const int n = min(128, g.nx + 2 - i0);
    const int t = threadIdx.x;
    if (n <= 0) return;
    tile_load<Q>(sf, f, g.cell(i0, j, k), n);
    tile_load<Q>(sg, fh, g.cell(i0, j, k), n);
    __syncthreads();
    if (t < n) {
        const long long c = g.cell(i0 + t, j, k);
        float tr = 0.f, tu = 0.f, tv = 0.f, tw = 0.f;
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            const float tf = sf[t * Q + l];
            tr += tf;
            macc(tu, lat_cx(l), tf);
            macc(tv, lat_cy(l), tf);
            macc(tw, lat_cz(l), tf);
        }
        const float inv = 1.0f / tr;
        const float ux = tu * inv, uy = tv * inv, uz = tw * inv;
        const float ax = uh[c] * inv, ay = vh[c] * inv, az = wh[c] * inv;
        const float base = rhoh[c] - (ax * ux + ay * uy + az * uz);
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            float d = base;
            macc(d, lat_cx(l), ax);
            macc(d, lat_cy(l), ay);
            macc(d, lat_cz(l), az);
            sg[t * Q + l] += d;
        }
    }
    __syncthreads();
    tile_store<Q>(sg, fh, g.cell(i0, j, k), n);
}

// Per-direction tables of the drift adjoints, in shared memory: a constant read
// indexed by l would serialise over the different directions of a warp.
template <int Q>
struct DriftTab {
    int cx[Q], cy[Q], cz[Q];
    long long d[Q];   // cell distance cx + (nx+2) cy + (nx+2)(ny+2) cz
};
template <int Q>
__device__ __forceinline__ void drift_tab(DriftTab<Q>& t, const RefGrid& g) {
    if (threadIdx.x < Q) {
        const int l = threadIdx.x;
        t.cx[l] = lat_cx(l);
        t.cy[l] = lat_cy(l);
        t.cz[l] = lat_cz(l);
        t.d[l] = lat_cx(l) + (long long)lat_cy(l) * (g.nx + 2) + (long long)lat_cz(l) * (g.nx + 2) * (g.ny + 2);
    }
    __syncthreads();
}
#define DRIFT_ADJ_ILP 4

// drift adjoint: fh_in(l, y) += fh_out(l, y + c_l) for y + c_l interior (the
// transpose of the pull).  One block per row (j,k) of the ghost-inclusive grid,
// looping over its (nx+2)*Q entries, DRIFT_ADJ_ILP loads in flight per thread.
template <int Q>
__global__ void __launch_bounds__(256) k_ref_drift_adj(float* __restrict__ fh_in, const float* __restrict__ fh_out,
                                                       RefGrid g) {
    __shared__ DriftTab<Q> t;
    drift_tab<Q>(t, g);
    const int j = blockIdx.x, k = blockIdx.y;
    const long long c0 = g.cell(0, j, k);
    const int n = Q * (g.nx + 2);
    for (int e0 = threadIdx.x; e0 < n; e0 += blockDim.x * DRIFT_ADJ_ILP) {
        float val[DRIFT_ADJ_ILP];
        bool ok[DRIFT_ADJ_ILP];
#pragma unroll
        for (int u = 0; u < DRIFT_ADJ_ILP; ++u) {
            const int e = e0 + u * blockDim.x;
            ok[u] = false;
            if (e >= n) continue;
            const int l = e % Q, i = e / Q;
            const int ti = i + t.cx[l], tj = j + t.cy[l], tk = k + t.cz[l];
            if (ti < 1 || ti > g.nx || tj < 1 || tj > g.ny || tk < 1 || tk > g.nz) continue;
            ok[u] = true;
            val[u] = fh_in[c0 * Q + e] + fh_out[(c0 + i + t.d[l]) * Q + l];
        }
#pragma unroll
        for (int u = 0; u < DRIFT_ADJ_ILP; ++u)
            if (ok[u]) fh_in[c0 * Q + e0 + u * blockDim.x] = val[u];
    }
}

// The macrovars adjoint at a cell x, as four terms: with a = (uh, vh, wh) / rho,
// d(rho, u)/df_l^T (rhoh, uh, vh, wh) = (rhoh - a.u) + a.c_l.  One thread per
// interior cell; T is [4][cells of the ghost-inclusive grid].
__global__ void __launch_bounds__(256) k_ref_macro_adj_terms(float* __restrict__ T, const float* __restrict__ rhoh,
                                                             const float* __restrict__ uh, const float* __restrict__ vh,
                                                             const float* __restrict__ wh, const float* __restrict__ rho,
                                                             const float* __restrict__ u, const float* __restrict__ v,
                                                             const float* __restrict__ w, RefGrid g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y + 1, k = blockIdx.z + 1;
    if (i > g.nx) return;
    const long long x = g.cell(i, j, k), n = g.ncell();
    const float inv = 1.0f / rho[x];
    const float ax = uh[x] * inv, ay = vh[x] * inv, az = wh[x] * inv;
    T[x] = rhoh[x] - (ax * u[x] + ay * v[x] + az * w[x]);
    T[n + x] = ax;
    T[2 * n + x] = ay;
    T[3 * n + x] = az;
}

// drift adjoint preceded by the adjoint of the macrovars call that followed the
// drift: fh_in(l, y) += fh_out(l, x) + d(rho, u)(x)/df_l^T (rhoh, uh, vh, wh)(x)
// for x = y + c_l interior, where rho(x), u(x) are the macrovars outputs and T
// holds the four terms of k_ref_macro_adj_terms.  The macrovars adjoints are
// taken at interior cells only.  Layout and loop as k_ref_drift_adj.
template <int Q>
__global__ void __launch_bounds__(256) k_ref_macro_drift_adj(float* __restrict__ fh_in,
                                                             const float* __restrict__ fh_out,
                                                             const float* __restrict__ T, RefGrid g) {
    __shared__ DriftTab<Q> t;
    drift_tab<Q>(t, g);
    const int j = blockIdx.x, k = blockIdx.y;
    const long long c0 = g.cell(0, j, k), nc = g.ncell();
    const int n = Q * (g.nx + 2);
    for (int e0 = threadIdx.x; e0 < n; e0 += blockDim.x * DRIFT_ADJ_ILP) {
        float val[DRIFT_ADJ_ILP];
        bool ok[DRIFT_ADJ_ILP];
#pragma unroll
        for (int q = 0; q < DRIFT_ADJ_ILP; ++q) {
            const int e = e0 + q * blockDim.x;
            ok[q] = false;
            if (e >= n) continue;
            const int l = e % Q, i = e / Q;
            const int cx = t.cx[l], cy = t.cy[l], cz = t.cz[l];
            const int ti = i + cx, tj = j + cy, tk = k + cz;
            if (ti < 1 || ti > g.nx || tj < 1 || tj > g.ny || tk < 1 || tk > g.nz) continue;
            ok[q] = true;
            const long long x = c0 + i + t.d[l];
            const float m = T[x] + (T[nc + x] * (float)cx + T[2 * nc + x] * (float)cy + T[3 * nc + x] * (float)cz);
            val[q] = fh_in[c0 * Q + e] + (fh_out[x * Q + l] + m);
        }
#pragma unroll
        for (int q = 0; q < DRIFT_ADJ_ILP; ++q)
            if (ok[q]) fh_in[c0 * Q + e0 + q * blockDim.x] = val[q];
    }
}

// the interior of an adjoint array is consumed (drift overwrote it in the forward);
// one block per row (j,k) of the interior, looping over its nx*nl floats
__global__ void __launch_bounds__(256) k_ref_zero_interior(float* fh, RefGrid g) {
    float* row = fh + g.cell(1, blockIdx.x + 1, blockIdx.y + 1) * g.nl;
    const int n = g.nl * g.nx;
    for (int e = threadIdx.x; e < n; e += blockDim.x) row[e] = 0.0f;
}

// Accessor of the boundary adjoint: the forward copy this(ld,i,j,k) = s(ls,si,sj,sk)
// becomes s^(ls,si,sj,sk) += this^(ld,i,j,k); this^(ld,i,j,k) = 0.  Within one
// boundary kernel the copies have distinct sources, or share one only inside
// the same thread (the inflow ghosts of a direction and its opposite), so the
// accumulation needs no atomics; the kernels themselves run in reverse order.
struct AdjAcc {
    float* f;
    RefGrid g;
    __device__ __forceinline__ float* p(int l, int i, int j, int k) const { return f + g.cell(i, j, k) * g.nl + l; }
    __device__ __forceinline__ void cp(int ld, int i, int j, int k, const AdjAcc& s, int ls, int si, int sj,
                                       int sk) const {
        float* d = p(ld, i, j, k);
        const float v = *d;
        *d = 0.0f;
        *s.p(ls, si, sj, sk) += v;
    }
};

// reverse of k_inflow: outflow copies first (they ran last), then the inflow ghosts;
// uvelh(k) receives d fghost / d uvel(k) times the ghosts' adjoints (one atomic
// per warp; launch with blocks of 32 threads over j, one k per block row).
// Every value is loaded before the first store, so the accesses of a thread
// overlap instead of running one read-modify-write at a time.
template <int Q, typename Acc>
__global__ void __launch_bounds__(128) k_inflow_adj(Acc f, float* uvelh, float rho0, float cosd, float sind) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int k = blockIdx.y + 1;
    const int nx = f.g.nx;
    float uh = 0.f;
    if (j <= f.g.ny) {
        float vo[Q], vi[Q], on[Q], o1[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            vo[l] = *f.p(l, nx + 1, j, k);
            vi[l] = *f.p(l, 0, j, k);
            on[l] = *f.p(l, nx, j, k);
            o1[l] = (lat_cx(l) <= 0 && nx > 1) ? *f.p(l, 1, j, k) : 0.0f;
        }
        const float cs2 = 1.0f / 3.0f;
        float acc[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) acc[l] = 0.0f;
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            const int s = (lat_cx(l) <= 0) ? l : lat_opposite(l);   // fghost(s) was stored at ghost l
            acc[s] += vi[l];
            uh -= vi[l] * 2.0f * lat_w<Q>(s) * rho0 * ((float)lat_cx(s) * cosd + (float)lat_cy(s) * sind) / cs2;
        }
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            *f.p(l, nx + 1, j, k) = 0.0f;
            *f.p(l, 0, j, k) = 0.0f;
            // the outflow copy's source (nx) first, then the inflow's (1); one cell when nx = 1
            float a = on[l] + vo[l];
            if (nx == 1 && lat_cx(l) <= 0) a += acc[l];
            *f.p(l, nx, j, k) = a;
            if (nx > 1 && lat_cx(l) <= 0) *f.p(l, 1, j, k) = o1[l] + acc[l];
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) uh += __shfl_down_sync(0xffffffffu, uh, o);
    if ((threadIdx.x & 31) == 0 && uh != 0.0f) atomicAdd(uvelh + (k - 1), uh);
}

// reverse of k_periodic (same grid): both ghost planes of the axis pass their
// adjoints to the planes they were copied from; loads before stores.  skipj:
// leave out the ghost rows j = 0, ny+1 (an accessor that wraps j maps them onto
// rows ny, 1, which other threads handle).
template <typename Acc>
__global__ void k_periodic_adj(Acc a, int axis, int nl, int skipj) {
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int l = blockIdx.z;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (l >= nl) return;
    if (skipj && ((axis == 0 && (t == 0 || t == ny + 1)) || (axis == 2 && (s == 0 || s == ny + 1)))) return;
    int n;
    float *g0, *g1, *sn, *s1;     // ghost 0, ghost n+1, their sources n and 1
    if (axis == 0) {
        if (t > ny + 1) return;
        n = nx; g0 = a.p(l, 0, t, s); g1 = a.p(l, nx + 1, t, s); sn = a.p(l, nx, t, s); s1 = a.p(l, 1, t, s);
    } else if (axis == 1) {
        if (t > nx + 1) return;
        n = ny; g0 = a.p(l, t, 0, s); g1 = a.p(l, t, ny + 1, s); sn = a.p(l, t, ny, s); s1 = a.p(l, t, 1, s);
    } else {
        if (t > nx + 1) return;
        n = nz; g0 = a.p(l, t, s, 0); g1 = a.p(l, t, s, nz + 1); sn = a.p(l, t, s, nz); s1 = a.p(l, t, s, 1);
    }
    const float v0 = *g0, v1 = *g1, wn = *sn, w1 = *s1;
    *g0 = 0.0f;
    *g1 = 0.0f;
    if (n == 1) {
        *sn = wn + v0 + v1;
    } else {
        *sn = wn + v0;
        *s1 = w1 + v1;
    }
}

// reverse of k_closed (same grid): per pair, f1(m,G) = f2(l,G) and
// f1(l,G) = f1(l,S) become f2^(l,G) += f1^(m,G), f1^(l,S) += f1^(l,G) with the
// ghost adjoints zeroed.  The reflected directions m and the outgoing l are
// disjoint sets and S is interior, so all loads can precede the stores.
template <typename Acc>
__global__ void __launch_bounds__(128) k_closed_adj(Acc f1, Acc f2, int axis, FacePairs lo, FacePairs hi) {
    pdl_enter();
    const int nx = f1.g.nx, ny = f1.g.ny, nz = f1.g.nz;
    const int side = blockIdx.z;
    const FacePairs& fp = side ? hi : lo;
    const int a = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int b = blockIdx.y + 1;
    int i, j, k, pi, pj, pk;
    if (axis == 0) {
        if (a > ny) return;
        j = a; k = b; i = side ? nx + 1 : 0; pi = side ? nx : 1; pj = j; pk = k;
    } else if (axis == 1) {
        if (a > nx) return;
        i = a; k = b; j = side ? ny + 1 : 0; pj = side ? ny : 1; pi = i; pk = k;
    } else {
        if (a > nx) return;
        i = a; j = b; k = side ? nz + 1 : 0; pk = side ? nz : 1; pi = i; pj = j;
    }
    float wm[9], wl[9], a2[9], ws[9];
    float* ps[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        if (q >= fp.n) break;
        const int l = fp.l[q], m = fp.m[q];
        const int si = (axis == 0) ? pi : pi - fp.cx[q];
        const int sj = (axis == 1) ? pj : pj - fp.cy[q];
        const int sk = (axis == 2) ? pk : pk - fp.cz[q];
        ps[q] = f1.p(l, si, sj, sk);
        wm[q] = *f1.p(m, i, j, k);
        wl[q] = *f1.p(l, i, j, k);
        a2[q] = *f2.p(l, i, j, k);
        ws[q] = *ps[q];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        if (q >= fp.n) break;
        const int l = fp.l[q], m = fp.m[q];
        *f1.p(m, i, j, k) = 0.0f;
        *f1.p(l, i, j, k) = 0.0f;
        *f2.p(l, i, j, k) = a2[q] + wm[q];
        *ps[q] = ws[q] + wl[q];
    }
}

}  // namespace lbm
