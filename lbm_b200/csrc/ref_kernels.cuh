// ref_kernels.cuh -- per-call kernels on the reference layout
// f(nl,0:nx+1,0:ny+1,0:nz+1) (l fastest), one per reference subroutine.
//
// Cell-wise kernels stage a row chunk of 128 cells (128*nl contiguous values)
// through shared memory, so the global reads and writes are coalesced even
// though each cell's nl populations are contiguous; the per-cell math reads
// the staged values with an odd stride (nl = 19 or 27), free of bank
// conflicts for FP32.
//
// Every kernel takes the arithmetic type R as a template argument: float for
// the reference's default build, double for its DP build (the _f64 entry
// points), where -r8 makes every real, tiny() and eps double precision.
#pragma once

#include "collide.cuh"

namespace lbm {


// Equilibrium offsets feq_l - w_l (m_fequil3_kernel.F90:58-113 in closed form).
template <int Q, typename R>
__device__ __forceinline__ void equilibrium(R (&fe)[Q], R drho, R rho, R ux, R uy, R uz, bool cubic) {
    const R usq = ux * ux + uy * uy + uz * uz;
    const R R45 = R(4.5) * rho;
    const R R45o = cubic ? R45 : R(0.0);
    const R A0 = drho - R(1.5) * rho * usq;
    const R B0 = R(3.0) * rho - (cubic ? R45 * usq : R(0.0));
    fe[0] = lat_w<Q, R>(0) * A0;
#pragma unroll
    for (int l = 1; l < Q; l += 2) {
        const R w = lat_w<Q, R>(l);
        const R cu = cdot(lat_cx(l), lat_cy(l), lat_cz(l), ux, uy, uz);
        const R cu2 = cu * cu;
        const R E = w * (A0 + R45 * cu2);
        const R O = w * cu * (B0 + R45o * cu2);
        fe[l] = E + O;
        fe[l + 1] = E - O;
    }
}

// Regularized non-equilibrium R(fneq) from a2 = sum H2 fneq (all l, including rest).
template <int Q, typename R>
__device__ __forceinline__ void regularized(R (&out)[Q], const MomentsT<R>& m, R ux, R uy, R uz) {
    const R third = R(1.0) / R(3.0);
    const R axx = m.pxx - m.s0 * third, ayy = m.pyy - m.s0 * third, azz = m.pzz - m.s0 * third;
    const R axy = m.pxy, axz = m.pxz, ayz = m.pyz;
    const R tr = axx + ayy + azz;
    const R vx = axx * ux + axy * uy + axz * uz;
    const R vy = axy * ux + ayy * uy + ayz * uz;
    const R vz = axz * ux + ayz * uy + azz * uz;
    out[0] = lat_w<Q, R>(0) * R(4.5) * (-tr * third);
#pragma unroll
    for (int l = 1; l < Q; l += 2) {
        const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
        const R w = R(4.5) * lat_w<Q, R>(l);
        const R cu = cdot(cx, cy, cz, ux, uy, uz);
        R cac = R(0);
        macc(cac, cx * cx, axx);
        macc(cac, cy * cy, ayy);
        macc(cac, cz * cz, azz);
        macc(cac, cx * cy, R(2.0) * axy);
        macc(cac, cx * cz, R(2.0) * axz);
        macc(cac, cy * cz, R(2.0) * ayz);
        const R cau = cdot(cx, cy, cz, vx, vy, vz);
        const R E = w * (cac - tr * third);
        const R O = w * (cu * (R(3.0) * cac - tr) - R(2.0) * cau);
        out[l] = E + O;
        out[l + 1] = E - O;
    }
}

// Row-chunk staging: cells [i0, i0+n) of row (j,k), n <= 128.
#define TILE_ILP 8
template <int Q, typename R>
__device__ __forceinline__ void tile_load(R* __restrict__ sm, const R* __restrict__ f, long long cell0, int n) {
    // TILE_ILP independent loads in flight per thread before their shared-memory stores
    const R* src = f + cell0 * Q;
    const int m = n * Q, step = blockDim.x * TILE_ILP;
    for (int e0 = threadIdx.x; e0 < m; e0 += step) {
        R v[TILE_ILP];
#pragma unroll
        for (int u = 0; u < TILE_ILP; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < m) v[u] = src[e];
        }
#pragma unroll
        for (int u = 0; u < TILE_ILP; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < m) sm[e] = v[u];
        }
    }
}
template <int Q, typename R>
__device__ __forceinline__ void tile_store(const R* __restrict__ sm, R* __restrict__ f, long long cell0, int n) {
    R* dst = f + cell0 * Q;
    const int m = n * Q;
    for (int e = threadIdx.x; e < m; e += blockDim.x) dst[e] = sm[e];
}

// fequil3: feq on interior cells (m_fequil3_kernel.F90:7-123)
template <int Q, typename R = float>
__global__ void __launch_bounds__(128) k_ref_fequil3(R* feq, const R* rho, const R* u, const R* v,
                                                     const R* w, RefGrid g, int ibgk) {
    __shared__ R sm[128 * Q];
    const int i0 = blockIdx.x * 128 + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
    const int n = min(128, g.nx + 1 - i0);
    const int t = threadIdx.x;
    if (n <= 0) return;
    if (t < n) {
        const long long c = g.cell(i0 + t, j, k);
        R fe[Q];
        equilibrium<Q>(fe, rho[c] - R(1.0), rho[c], u[c], v[c], w[c], ibgk == 3);
#pragma unroll
        for (int l = 0; l < Q; ++l) sm[t * Q + l] = fe[l] + lat_w<Q, R>(l);
    }
    __syncthreads();
    tile_store<Q>(sm, feq, g.cell(i0, j, k), n);
}

// postcoll: collide interior cells in place with the given moments (m_postcoll_kernel.F90:7-255)
template <int Q, typename R = float>
__global__ void __launch_bounds__(128) k_ref_postcoll(R* f, R* tau, const R* rho, const R* u,
                                                      const R* v, const R* w, const R* abl, RefGrid g,
                                                      CollideParamsT<R> cp) {
    __shared__ R sm[128 * Q];
    const int i0 = blockIdx.x * 128 + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
    const int n = min(128, g.nx + 1 - i0);
    const int t = threadIdx.x;
    if (n <= 0) return;
    tile_load<Q>(sm, f, g.cell(i0, j, k), n);
    __syncthreads();
    if (t < n) {
        const long long c = g.cell(i0 + t, j, k);
        R fp[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) fp[l] = sm[t * Q + l] - lat_w<Q, R>(l);
        const MomentsT<R> m = moments<Q>(fp);
        const R r = rho[c];
        TurbInT<R> tb;
        tb.on = false;
        tb.dux = tb.duy = tb.duz = R(0);
        const R tnew = collide<Q>(fp, m, r - R(1.0), r, u[c], v[c], w[c], cp, abl ? abl[k - 1] : R(0.0), tau[c],
                                      false, tb);
        if (cp.ivreman) tau[c] = tnew;
#pragma unroll
        for (int l = 0; l < Q; ++l) sm[t * Q + l] = fp[l] + lat_w<Q, R>(l);
    }
    __syncthreads();
    tile_store<Q>(sm, f, g.cell(i0, j, k), n);
}

// drift: f(l,i,j,k) = feq(l,i-cx,j-cy,k-cz) over interior cells; a thread per
// (l,i) of a row, as m_drift_kernel.F90:33-42 flattens it.  The source of
// element e = (i-1) Q + l of a row is e minus the direction's distance Q d_l,
// d_l = cx + (nx+2) cy + (nx+2)(ny+2) cz, taken from shared memory (a constant
// read would serialise over the different l of a warp).  Each thread keeps
// DRIFT_ILP loads in flight before its stores.
#define DRIFT_ILP 4
template <int Q, typename R = float>
__global__ void __launch_bounds__(256) k_ref_drift(R* __restrict__ f, const R* __restrict__ feq, RefGrid g) {
    // one block per interior row (j,k), looping over its nx*Q outputs
    __shared__ long long sd[Q];
    if (threadIdx.x < Q) {
        const int l = threadIdx.x;
        sd[l] = (long long)Q * (lat_cx(l) + (long long)lat_cy(l) * (g.nx + 2) +
                                (long long)lat_cz(l) * (g.nx + 2) * (g.ny + 2));
    }
    __syncthreads();
    const int j = blockIdx.x + 1, k = blockIdx.y + 1;
    const long long base = g.cell(1, j, k) * Q;
    const int n = Q * g.nx;
    for (int e0 = threadIdx.x; e0 < n; e0 += blockDim.x * DRIFT_ILP) {
        R v[DRIFT_ILP];
#pragma unroll
        for (int u = 0; u < DRIFT_ILP; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < n) v[u] = feq[base + e - sd[e % Q]];
        }
#pragma unroll
        for (int u = 0; u < DRIFT_ILP; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < n) f[base + e] = v[u];
        }
    }
}

// macrovars over the ghost-inclusive grid, summation order of m_macrovars_kernel.F90:35-49
template <int Q, typename R = float>
__global__ void __launch_bounds__(128) k_ref_macrovars(R* rho, R* u, R* v, R* w, const R* f,
                                                       RefGrid g) {
    __shared__ R sm[128 * Q];
    const int i0 = blockIdx.x * 128, j = blockIdx.y, k = blockIdx.z;
    const int n = min(128, g.nx + 2 - i0);
    const int t = threadIdx.x;
    if (n <= 0) return;
    tile_load<Q>(sm, f, g.cell(i0, j, k), n);
    __syncthreads();
    if (t < n) {
        R tr = R(0), tu = R(0), tv = R(0), tw = R(0);
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            const R tf = sm[t * Q + l];
            tr = tr + tf;
            macc(tu, lat_cx(l), tf);
            macc(tv, lat_cy(l), tf);
            macc(tw, lat_cz(l), tf);
        }
        const R inv = R(1.0) / tr;
        const long long c = g.cell(i0 + t, j, k);
        rho[c] = tr;
        u[c] = tu * inv;
        v[c] = tv * inv;
        w[c] = tw * inv;
    }
}

// regularization: f = R(f - feq) on interior cells (m_regularization_kernel.F90:6-122)
template <int Q, typename R = float>
__global__ void __launch_bounds__(128) k_ref_regularization(R* f, const R* feq, const R* u,
                                                            const R* v, const R* w, RefGrid g) {
    __shared__ R sm[128 * Q];
    const int i0 = blockIdx.x * 128 + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
    const int n = min(128, g.nx + 1 - i0);
    const int t = threadIdx.x;
    if (n <= 0) return;
    tile_load<Q>(sm, f, g.cell(i0, j, k), n);
    __syncthreads();
    if (t < n) {
        const long long c = g.cell(i0 + t, j, k);
        R fn[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) fn[l] = sm[t * Q + l] - feq[c * Q + l];
        const MomentsT<R> m = moments<Q>(fn);
        R out[Q];
        regularized<Q>(out, m, u[c], v[c], w[c]);
#pragma unroll
        for (int l = 0; l < Q; ++l) sm[t * Q + l] = out[l];
    }
    __syncthreads();
    tile_store<Q>(sm, f, g.cell(i0, j, k), n);
}

// vreman: tau from a non-equilibrium f with the standalone guards
// (alphamag and beta start at 1e-5, no ablvisc; m_vreman_kernel.F90:47-91)
template <int Q, typename R = float>
__global__ void __launch_bounds__(128) k_ref_vreman(const R* f, R* tau, RefGrid g, CollideParamsT<R> cp) {
    __shared__ R sm[128 * Q];
    const int i0 = blockIdx.x * 128 + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
    const int n = min(128, g.nx + 1 - i0);
    const int t = threadIdx.x;
    if (n <= 0) return;
    tile_load<Q>(sm, f, g.cell(i0, j, k), n);
    __syncthreads();
    if (t < n) {
        R fn[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) fn[l] = sm[t * Q + l];
        const MomentsT<R> m = moments<Q>(fn);
        const R third = R(1.0) / R(3.0);
        const R axx = m.pxx - m.s0 * third, ayy = m.pyy - m.s0 * third, azz = m.pzz - m.s0 * third;
        const R axy = m.pxy, axz = m.pxz, ayz = m.pyz;
        const R g0 = R(0.00001);
        const R amag = g0 + (axx * axx + ayy * ayy + azz * azz + R(2.0) * (axy * axy + axz * axz + ayz * ayz));
        const R b11 = g0 + axx * axx + axy * axy + axz * axz;
        const R b22 = g0 + axy * axy + ayy * ayy + ayz * ayz;
        const R b33 = g0 + axz * axz + ayz * ayz + azz * azz;
        const R b12 = g0 + axx * axy + axy * ayy + axz * ayz;
        const R b13 = g0 + axx * axz + axy * ayz + axz * azz;
        const R b23 = g0 + axy * axz + ayy * ayz + ayz * azz;
        const R bb = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
        const R tt = bb / amag;
        const R nut = (tt > cp.eps) ? cp.cvre * real_sqrt(tt) : R(0.0);
        tau[g.cell(i0 + t, j, k)] = R(3.0) * (cp.kinevisc + nut) + R(0.5);
    }
}

// compute_fneq / compute_f: elementwise over every element, ghosts included
template <typename R = float>
__global__ void k_ref_axpy(R* f, const R* feq, long long n, int sgn) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        f[e] = (sgn > 0) ? (feq[e] + f[e]) : (f[e] - feq[e]);
}

// solids: swap pairs (l,l+1), l = 2,4,..,nl-1 (1-based) at blanked interior cells (m_solids.F90:24-36)
template <int Q, typename R = float>
__global__ void k_ref_solids(R* f, const int32_t* blank, RefGrid g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
    if (i > g.nx) return;
    const long long c = g.cell(i, j, k);
    if (blank[c] == 0) return;
    R* p = f + c * Q;
#pragma unroll
    for (int l = 1; l + 1 < Q; l += 2) {
        const R a = p[l];
        p[l] = p[l + 1];
        p[l + 1] = a;
    }
}

// forcings_apply: f += feq2(rho, u - F/rho) - feq2(rho, u) at interior cells with
// rho > 0 (m_forcings_apply_kernel.F90:47-213; second-order equilibria), in the
// closed form w rho [3 dcu + 4.5 dcu (2 cu + dcu) - 1.5 (2 u.du + du.du)].
template <int Q, typename R = float>
__global__ void __launch_bounds__(128) k_ref_forcings_apply(R* f, const R* force, const R* rho,
                                                            const R* u, const R* v, const R* w, RefGrid g) {
    __shared__ R sm[128 * Q];
    const int i0 = blockIdx.x * 128 + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
    const int n = min(128, g.nx + 1 - i0);
    const int t = threadIdx.x;
    if (n <= 0) return;
    tile_load<Q>(sm, f, g.cell(i0, j, k), n);
    __syncthreads();
    if (t < n) {
        const long long c = g.cell(i0 + t, j, k);
        const R rr = rho[c];
        if (rr > R(0.0)) {
            const R ux = u[c], uy = v[c], uz = w[c];
            const R dux = -force[3 * c] / rr, duy = -force[3 * c + 1] / rr, duz = -force[3 * c + 2] / rr;
            const R dusq = dux * (R(2.0) * ux + dux) + duy * (R(2.0) * uy + duy) + duz * (R(2.0) * uz + duz);
            R* p = sm + t * Q;
            p[0] += lat_w<Q, R>(0) * rr * (-R(1.5) * dusq);
#pragma unroll
            for (int l = 1; l < Q; l += 2) {
                const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
                const R cu = cdot(cx, cy, cz, ux, uy, uz);
                const R dcu = cdot(cx, cy, cz, dux, duy, duz);
                const R wr = lat_w<Q, R>(l) * rr;
                const R dE = wr * (R(4.5) * dcu * (R(2.0) * cu + dcu) - R(1.5) * dusq);
                const R dO = wr * R(3.0) * dcu;
                p[l] += dE + dO;
                p[l + 1] += dE - dO;
            }
        }
    }
    __syncthreads();
    tile_store<Q>(sm, f, g.cell(i0, j, k), n);
}

// inflow_turbulence_forcing: df(l,j,k) = feq(rho,u+ampl*uu) - feq(rho,u) at i = iturb
// (m_inflow_turbulence_forcing.F90:44-128), evaluated as a difference of offsets
template <int Q, typename R = float>
__global__ void k_ref_turb_forcing(R* df, const R* rho, const R* u, const R* v, const R* w,
                                   const R* uu, const R* vv, const R* ww, R ampl, int lit, int ip,
                                   int ibgk, RefGrid g) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1, k = blockIdx.y + 1;
    if (j > g.ny) return;
    const long long c = g.cell(ip, j, k);
    const long long t = (long long)(j - 1) + (long long)g.ny * ((long long)(k - 1) + (long long)g.nz * lit);
    const R r = rho[c];
    const R ux = u[c], uy = v[c], uz = w[c];
    const R dux = ampl * uu[t], duy = ampl * vv[t], duz = ampl * ww[t];
    const bool cubic = ibgk == 3;
    const R usq = ux * ux + uy * uy + uz * uz;
    const R dusq = dux * (R(2.0) * ux + dux) + duy * (R(2.0) * uy + duy) + duz * (R(2.0) * uz + duz);
    const R usq2 = usq + dusq;
    R* o = df + ((long long)(j - 1) + (long long)g.ny * (k - 1)) * Q;
    o[0] = lat_w<Q, R>(0) * r * (-R(1.5) * dusq);
#pragma unroll
    for (int l = 1; l < Q; l += 2) {
        const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
        const R wr = lat_w<Q, R>(l) * r;
        const R cu = cdot(cx, cy, cz, ux, uy, uz);
        const R dcu = cdot(cx, cy, cz, dux, duy, duz);
        const R cun = cu + dcu;
        const R E = wr * (R(4.5) * dcu * (R(2.0) * cu + dcu) - R(1.5) * dusq);
        R od = R(3.0) * dcu;
        if (cubic) od += R(4.5) * dcu * (cun * cun + cun * cu + cu * cu - usq2) - R(4.5) * cu * dusq;
        const R O = wr * od;
        o[l] = E + O;
        o[l + 1] = E - O;
    }
}

// inflow_turbulence_apply: f(l,ip,j,k) += df(l,j,k) (m_inflow_turbulence_apply.F90:19-28)
template <typename R = float>
__global__ void k_ref_turb_apply(R* f, const R* df, int ip, RefGrid g) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;   // over (l, j)
    const int k = blockIdx.y + 1;
    const int nl = g.nl;
    if (e >= nl * g.ny) return;
    const int l = e % nl, j = e / nl + 1;
    f[g.cell(ip, j, k) * nl + l] += df[((long long)(j - 1) + (long long)g.ny * (k - 1)) * nl + l];
}

// fillghosts: ghost cells copy the nearest interior cell (m_fillghosts.F90:18-29)
template <typename R = float>
__global__ void k_ref_fillghosts(R* f, RefGrid g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i > g.nx + 1) return;
    const int i1 = min(max(i, 1), g.nx), j1 = min(max(j, 1), g.ny), k1 = min(max(k, 1), g.nz);
    if (i1 == i && j1 == j && k1 == k) return;
    const int nl = g.nl;
    const R* s = f + g.cell(i1, j1, k1) * nl;
    R* d = f + g.cell(i, j, k) * nl;
    for (int l = 0; l < nl; ++l) d[l] = s[l];
}

}  // namespace lbm
