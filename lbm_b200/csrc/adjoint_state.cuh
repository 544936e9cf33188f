// adjoint_state.cuh -- the reverse sweep in the state (structure-of-arrays)
// layout, for forward runs made with the fused step.
//
// The adjoints are FP32 arrays with the fused state's geometry (SoaGrid) and
// an explicit ghost shell, i.e. the reference-layout arrays f1^, f2^ stored as
// structure of arrays.  One reverse step is the per-call chain of adjoint.cuh
// (drift, boundarycond, solids, postcoll, macrovars) with two differences: the
// forward pre-collision populations are pulled from a copy of the fused state
// buffer of the previous step, and the moments are those of the populations
// themselves (the fused step takes rho, u from f), so the macrovars adjoint is
// part of the cell kernel.  All accesses are coalesced: the transpose of the
// pull is a shift by +c_l of each direction's block.
#pragma once

#include <algorithm>

#include "adjoint.cuh"
#include "state_kernels.cuh"

namespace lbm {

// boundary adjoint accessor on a state-layout FP32 array with explicit ghosts.
// wrap (periodic j): the ghost rows j = 0 and ny+1 are rows ny and 1, as in the
// fused forward state, so the periodic copies are identities and never run.
struct SoaAdjAcc {
    float* f;
    SoaGrid g;
    int wrap;
    __device__ __forceinline__ float* p(int l, int i, int j, int k) const {
        return f + (long long)l * g.dstride + g.off(i, wrap ? wrapj(j, g.ny) : j, k);
    }
    __device__ __forceinline__ void cp(int ld, int i, int j, int k, const SoaAdjAcc& s, int ls, int si, int sj,
                                       int sk) const {
        float* d = p(ld, i, j, k);
        const float v = *d;
        *d = 0.0f;
        *s.p(ls, si, sj, sk) += v;
    }
};

__device__ __forceinline__ bool interior(const SoaGrid& g, int i, int j, int k) {
    return i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
}

// the ghost shell and the interior cells next to it: the only cells whose
// adjoint entries the boundary adjoint reads or writes (with wrap, j plays no part)
__device__ __forceinline__ bool near_shell(const SoaGrid& g, int i, int j, int k, bool wrap) {
    return i <= 1 || i >= g.nx || (!wrap && (j <= 1 || j >= g.ny)) || k <= 1 || k >= g.nz;
}

// element distance from cell (i,j,k) to (i+cx, j+cy, k+cz) of direction l; with
// wrap, a target row 0 or ny+1 is row ny or 1
__device__ __forceinline__ long long push_delta(const SoaGrid& g, int l, int j, bool wrap) {
    const long long rs = g.pitch, ps = (long long)g.pitch * (g.ny + 2);
    long long d = lat_cx(l) + lat_cy(l) * rs + lat_cz(l) * ps;
    if (wrap) {
        if (lat_cy(l) < 0 && j == 1) d += (long long)g.ny * rs;
        if (lat_cy(l) > 0 && j == g.ny) d -= (long long)g.ny * rs;
    }
    return d;
}

// the k-th of the distinct values {0, 1, n, n+1} (count: min(4, n + 2))
__device__ __forceinline__ int edge_value(int idx, int n) {
    const int cnt = min(4, n + 2);
    return idx < 2 ? idx : n + 2 - cnt + idx;
}

// Before the boundary adjoint.  (1) The drift transpose for ghost targets:
// W(l, y) += A(l, y + c_l) for ghost cells y whose target y + c_l is interior.
// (2) W(l, y) = 0 at the interior cells next to the shell: the interior of f2
// is overwritten by the next step's collision, so its adjoint is zero before
// the boundary adjoint accumulates into it.  Interior elements of A are read,
// not cleared; the cell kernel reads each of the others exactly once.
// A thread per cell of the two outer layers: first the whole rows (j, k) with
// k in {0, 1, nz, nz+1} or (without wrap) j in {0, 1, ny, ny+1} (coalesced), then
// the cells i in {0, 1, nx, nx+1} of the other rows.  With wrap only the rows
// j = 1..ny exist.
template <int Q>
__global__ void __launch_bounds__(128) k_sadj_shell(float* __restrict__ W, const float* __restrict__ A, SoaGrid g,
                                                    int wrap) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int ck = min(4, nz + 2), cj = wrap ? 0 : min(4, ny + 2), cx = min(4, nx + 2);
    const int kin = max(0, nz - 2), jin = wrap ? ny : max(0, ny - 2), j0 = wrap ? 1 : 2;
    const int nj = wrap ? ny : ny + 2;        // rows of a k-shell plane
    const long long full_rows = (long long)ck * nj + (long long)cj * kin;
    const long long nfull = full_rows * (nx + 2);
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (t < nfull) {
        const long long r = t / (nx + 2);
        i = (int)(t - r * (nx + 2));
        if (r < (long long)ck * nj) {
            k = edge_value((int)(r / nj), nz);
            j = (int)(r % nj) + (wrap ? 1 : 0);
        } else {
            const int q = (int)(r - (long long)ck * nj);
            j = edge_value(q / kin, ny);
            k = 2 + q % kin;
        }
    } else {
        const long long u = t - nfull;
        if (u >= (long long)jin * kin * cx) return;
        const int r = (int)(u / cx);
        i = edge_value((int)(u - (long long)r * cx), nx);
        j = j0 + r % jin;
        k = 2 + r / jin;
    }
    const long long o = g.off(i, j, k);
    if (interior(g, i, j, k)) {
#pragma unroll
        for (int l = 0; l < Q; ++l) W[(long long)l * g.dstride + o] = 0.0f;
        return;
    }
    float v[Q], w[Q];
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        const int jt = wrap ? wrapj(j + lat_cy(l), ny) : j + lat_cy(l);
        v[l] = interior(g, i + lat_cx(l), jt, k + lat_cz(l)) ? A[(long long)l * g.dstride + o + push_delta(g, l, j, wrap)]
                                                               : 0.0f;
        w[l] = W[(long long)l * g.dstride + o];
    }
#pragma unroll
    for (int l = 0; l < Q; ++l) W[(long long)l * g.dstride + o] = w[l] + v[l];
}

// threads of k_sadj_shell
inline long long sadj_shell_cells(const SoaGrid& g, bool wrap) {
    const long long ck = std::min(4, g.nz + 2), cj = wrap ? 0 : std::min(4, g.ny + 2), cx = std::min(4, g.nx + 2);
    const long long kin = std::max(0, g.nz - 2), jin = wrap ? g.ny : std::max(0, g.ny - 2);
    const long long nj = wrap ? g.ny : g.ny + 2;
    return (ck * nj + cj * kin) * (g.nx + 2) + jin * kin * cx;
}

// ---- the folded configuration (inflow/outflow i, periodic j read as rows ny and
// 1, closed k): the shell and the inflow adjoint without strided passes over Q ----

// Shell of the folded configuration without its x faces: the k ghost rows
// (k = 0, nz+1, j = 1..ny, every i) take the drift transpose of their ghost
// targets, and W = 0 at the cells i = 2..nx-1 of the rows k = 1, nz.  The x
// faces (i = 0, 1, nx, nx+1 of the rows k = 1..nz) are k_sadj_xface's.
template <int Q>
__global__ void __launch_bounds__(128) k_sadj_shell_fold(float* __restrict__ W, const float* __restrict__ A, SoaGrid g) {
    pdl_enter();
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long nghost = 2LL * ny * (nx + 2);
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nghost) {
        const long long r = t / (nx + 2);
        const int i = (int)(t - r * (nx + 2));
        const int j = 1 + (int)(r % ny);
        const int k = (r < ny) ? 0 : nz + 1;
        const long long o = g.off(i, j, k);
        float v[Q], w[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            const int it = i + lat_cx(l), kt = k + lat_cz(l);
            v[l] = (it >= 1 && it <= nx && kt >= 1 && kt <= nz) ? A[(long long)l * g.dstride + o + push_delta(g, l, j, true)]
                                                               : 0.0f;
            w[l] = W[(long long)l * g.dstride + o];
        }
#pragma unroll
        for (int l = 0; l < Q; ++l) W[(long long)l * g.dstride + o] = w[l] + v[l];
        return;
    }
    const int nkr = (nz > 1) ? 2 : 1, ni = nx - 2;
    const long long u = t - nghost;
    if (ni <= 0 || u >= (long long)nkr * ny * ni) return;
    const long long r = u / ni;
    const int i = 2 + (int)(u - r * ni);
    const int j = 1 + (int)(r % ny);
    const int k = (r < ny) ? 1 : nz;
    const long long o = g.off(i, j, k);
#pragma unroll
    for (int l = 0; l < Q; ++l) W[(long long)l * g.dstride + o] = 0.0f;
}
inline long long sadj_shell_fold_cells(const SoaGrid& g) {
    return 2LL * g.ny * (g.nx + 2) + (long long)((g.nz > 1) ? 2 : 1) * g.ny * std::max(0, g.nx - 2);
}

// The x faces of the folded configuration, rows k = 1..nz: the drift transpose
// for the x ghosts, then the reverse of the outflow copy and of the inflow
// ghosts (k_inflow_adj), one thread per (direction, j, k).  The adjoints at the
// cells i = 1 and nx are written, not accumulated: nothing earlier in the
// reverse step reaches them.  The inflow ghost of a direction l with cx > 0 is
// its opposite's corrected value, so the thread of a direction s with cx < 0
// also consumes the ghost adjoint of opp(s).  Between the rows k = 2 and nz-1
// the x-ghost adjoints are zero when this kernel runs (only the closed-k adjoint
// adds to x ghosts, and only in the rows 1 and nz), so there they are neither
// read nor cleared.  Grid: x over j (32 per block), y = direction, z = k;
// uvelh(k) gets one atomic per warp.
template <int Q>
__global__ void __launch_bounds__(32) k_sadj_xface(float* __restrict__ W, const float* __restrict__ A, SoaGrid g,
                                                   float* __restrict__ uvelh, float rho0, float cosd, float sind) {
    pdl_enter();
    const int j = blockIdx.x * 32 + threadIdx.x + 1;
    const int l = blockIdx.y, k = blockIdx.z + 1;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    float uh = 0.0f;
    if (j <= ny) {
        const int cx = c_cx[l], cy = c_cy[l], cz = c_cz[l];
        const long long dl = (long long)l * g.dstride;
        const long long o0 = g.off(0, j, k), on = g.off(nx, j, k);
        const bool kface = (k == 1 || k == nz);      // x-ghost adjoints may be nonzero
        // outflow: f(l, nx+1) = f(l, nx); the ghost's adjoint includes its pull (cx < 0)
        float vo = kface ? W[dl + on + 1] : 0.0f;
        if (cx < 0 && k + cz >= 1 && k + cz <= nz)
            vo += A[dl + g.off(nx, wrapj(j + cy, ny), k + cz)];
        // inflow ghosts at i = 0 whose source is direction l (cx <= 0): l itself and, for cx < 0, opp(l)
        float acc = 0.0f, vi = 0.0f, vp = 0.0f;
        int lo = l;
        if (cx <= 0) {
            if (kface) vi = W[dl + o0];
            if (cx < 0) {
                lo = c_opp[l];
                const long long dlo = (long long)lo * g.dstride;
                if (kface) vp = W[dlo + o0];
                if (k - cz >= 1 && k - cz <= nz) vp += A[dlo + g.off(1, wrapj(j - cy, ny), k - cz)];
            }
            acc = vi + vp;
        }
        if (kface) {
            W[dl + on + 1] = 0.0f;
            if (cx <= 0) W[dl + o0] = 0.0f;
            if (cx < 0) W[(long long)lo * g.dstride + o0] = 0.0f;
        }
        W[dl + on] = vo;
        if (cx <= 0) {
            const float wl = c_w[Q == 27 ? 1 : 0][l];
            uh = -acc * 2.0f * wl * rho0 * ((float)cx * cosd + (float)cy * sind) * 3.0f;
        }
        W[dl + g.off(1, j, k)] = acc;    // zero for cx > 0: no inflow ghost comes from l
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) uh += __shfl_down_sync(0xffffffffu, uh, o);
    if (threadIdx.x == 0 && uh != 0.0f) atomicAdd(uvelh + (k - 1), uh);
}

// One reverse step at the interior cells: the drift transpose for interior
// targets, gh(l, y) = A(l, y + c_l) (+ W(l, y), the boundary adjoint's
// contributions, next to the shell), then the postcoll (+solids, +the
// macrovars of its input) adjoint; W receives the adjoint of the pre-collision
// populations.  PULL: the forward input is pull(P) (P a copy of the previous
// step's fused state buffer, offsets f - w, FP32); otherwise it is P itself
// (the state as imported).  wrap: P has periodic j without stored ghost rows;
// awrap: the adjoint arrays read their j ghost rows as rows ny and 1 (SoaAdjAcc).
// ROWS: the row is j = 1 or ny, where periodic j wraps (otherwise the wrap
// adjustments of every address are compiled out).
template <int Q, bool PULL, bool ROWS>
__device__ __forceinline__ void sadj_cell(float* __restrict__ W, const float* __restrict__ A,
                                          const float* __restrict__ P, const SoaGrid& g, int wrap_, int awrap_,
                                          const uint8_t* __restrict__ solid, const CollideParams& cp,
                                          const float* __restrict__ abl, int i, int j, int k) {
    const int wrap = ROWS ? wrap_ : 0, awrap = ROWS ? awrap_ : 0;
    const long long o = g.off(i, j, k);
    float fp[Q], gh[Q];
    if (PULL) {
        PullMacro<Q, float, 0>::run(fp, P, g, o, j, wrap != 0);
    } else {
#pragma unroll
        for (int l = 0; l < Q; ++l) fp[l] = P[(long long)l * g.dstride + o];
    }
    const bool wr = awrap != 0;
#pragma unroll
    for (int l = 0; l < Q; ++l) gh[l] = A[(long long)l * g.dstride + o + push_delta(g, l, j, wr)];
    if (near_shell(g, i, j, k, wr)) {
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            const int jt = wr ? wrapj(j + lat_cy(l), g.ny) : j + lat_cy(l);
            gh[l] = (interior(g, i + lat_cx(l), jt, k + lat_cz(l)) ? gh[l] : 0.0f) + W[(long long)l * g.dstride + o];
        }
    }
    if (solid && solid[((long long)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1)]) {
#pragma unroll
        for (int l = 1; l + 1 < Q; l += 2) {
            const float x = gh[l];
            gh[l] = gh[l + 1];
            gh[l + 1] = x;
        }
    }
    const Moments m = moments_rows<Q>(fp);
    const float rho = 1.0f + m.s0;
    const float irho = 1.0f / rho;
    const float ux = m.jx * irho, uy = m.jy * irho, uz = m.jz * irho;
    float rh = 0.f, uxh = 0.f, uyh = 0.f, uzh = 0.f;
    const CollideAdjOut c = collide_adj_moments<Q>(m, gh, rho, ux, uy, uz, cp, abl ? abl[k - 1] : 0.0f, cp.tau0, rh,
                                                   uxh, uyh, uzh);
    // rho = sum f, u = (sum c f) / rho; the adjoint of f_l is E +- O over the
    // opposite pair (l, l+1): E = s0h + rh - a.u + c c : a_h, O = c . a
    const float ax = uxh * irho, ay = uyh * irho, az = uzh * irho;
    const float E0 = c.s0h + rh - (ax * ux + ay * uy + az * uz);
    W[o] = E0;
#pragma unroll
    for (int l = 1; l < Q; l += 2) {
        const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
        float E = E0, O = 0.0f;
        macc(E, cx * cx, c.axxh);
        macc(E, cy * cy, c.ayyh);
        macc(E, cz * cz, c.azzh);
        macc(E, cx * cy, c.axyh);
        macc(E, cx * cz, c.axzh);
        macc(E, cy * cz, c.ayzh);
        macc(O, cx, ax);
        macc(O, cy, ay);
        macc(O, cz, az);
        W[(long long)l * g.dstride + o] = E + O;
        W[(long long)(l + 1) * g.dstride + o] = E - O;
    }
}

template <int Q, bool PULL>
__global__ void __launch_bounds__(128) k_sadj_cell(float* __restrict__ W, const float* __restrict__ A,
                                                   const float* __restrict__ P, SoaGrid g, int wrap, int awrap,
                                                   const uint8_t* __restrict__ solid, CollideParams cp,
                                                   const float* __restrict__ abl) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y + 1, k = blockIdx.z + 1;
    if (i > g.nx) return;
    if (j == 1 || j == g.ny) sadj_cell<Q, PULL, true>(W, A, P, g, wrap, awrap, solid, cp, abl, i, j, k);
    else sadj_cell<Q, PULL, false>(W, A, P, g, wrap, awrap, solid, cp, abl, i, j, k);
}

// loss seed: A(l, x_p) += d(u, v, w)(x_p)/df_l^T uhat_p at the probe cells, where
// f = pull(P) is the reference's f1 after the last step.  probes: (i, j, k)
// triples, 1-based, distinct; uhat: (P, 3).
template <int Q>
__global__ void k_sadj_seed(float* A, const float* __restrict__ P, SoaGrid g, int wrap, const int* probes,
                            const float* uhat, int np) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const int i = probes[3 * p], j = probes[3 * p + 1], k = probes[3 * p + 2];
    const long long o = g.off(i, j, k);
    float fp[Q];
    PullMacro<Q, float, 0>::run(fp, P, g, o, j, wrap != 0);
    const Moments m = moments<Q>(fp);
    const float rho = 1.0f + m.s0;
    const float ux = m.jx / rho, uy = m.jy / rho, uz = m.jz / rho;
    const float ax = uhat[3 * p] / rho, ay = uhat[3 * p + 1] / rho, az = uhat[3 * p + 2] / rho;
    const float base = -(ax * ux + ay * uy + az * uz);
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        float d = base;
        macc(d, lat_cx(l), ax);
        macc(d, lat_cy(l), ay);
        macc(d, lat_cz(l), az);
        A[(long long)l * g.dstride + o] += d;
    }
}

// a state-layout adjoint to the reference layout (all cells, no weights: adjoints of
// f and of f - w are the same).  A block of 128 cells of one row is staged
// through shared memory, so both the reads (per direction, along i) and the
// writes (l fastest) are coalesced.  Grid: x over i in blocks of 128, y = j, z = k.
template <int Q>
__global__ void __launch_bounds__(128) k_sadj_export(float* __restrict__ ref, const float* __restrict__ A, SoaGrid g) {
    __shared__ float sm[128 * Q];
    const int i0 = blockIdx.x * 128;
    const int j = blockIdx.y, k = blockIdx.z;
    const int n = min(128, g.nx + 2 - i0);
    if (n <= 0) return;
    const int t = threadIdx.x;
    if (t < n) {
        const long long o = g.off(i0 + t, j, k);
#pragma unroll
        for (int l = 0; l < Q; ++l) sm[t * Q + l] = A[(long long)l * g.dstride + o];
    }
    __syncthreads();
    const long long base = ((long long)i0 + (long long)(g.nx + 2) * ((long long)j + (long long)(g.ny + 2) * k)) * Q;
    for (int e = t; e < n * Q; e += blockDim.x) ref[base + e] = sm[e];
}

}  // namespace lbm
