// state_kernels.cuh -- kernels of the fused state (structure of arrays).
//
// One launch of k_step performs, for every interior cell, what the reference
// does in drift -> macrovars -> inflow_turbulence_forcing -> postcoll ->
// inflow_turbulence_apply -> solids (main.F90:322-329 of step n-1 and
// :296-310 of step n): it pulls the post-collision populations of the
// neighbours, forms the moments in registers, collides, and writes the new
// post-collision populations once.  The boundary ghost kernels then run in the
// reference's order on the new buffer, reading the old buffer's ghosts for
// the two-step bounce-back.
#pragma once

#include "collide.cuh"

namespace lbm {

struct StepArgs {
    SoaGrid g;
    CollideParams cp;
    const uint8_t* solid;     // interior mask [k-1][j-1][i-1], or null
    const float* uu;          // turbulence fields (ny,nz,0:nrturb) or null
    const float* vv;
    const float* ww;
    int nrturb;
    float ampl;
    int iturb;                // 1-based i of the forcing slice
    const int* d_it;          // number of the step being computed (device)
    const float* abl;         // ablvisc(nz) or null
    int* status;              // LBM_STATUS_* bits
    // collide-in-place mode: the moments postcoll uses come from these arrays
    const float* rho_in;      // reference layout (0:nx+1,0:ny+1,0:nz+1)
    const float* u_in;
    const float* v_in;
    const float* w_in;
};

__device__ __forceinline__ void flag_bad_density(int* status, float rho, float ux, float uy, float uz) {
    const float chk = rho + ux + uy + uz;
    const bool bad = !(rho > 0.0f) || !(fabsf(chk) < 1.0e30f);
    const unsigned mask = __activemask();
    const unsigned vote = __ballot_sync(mask, bad);
    if (vote && (threadIdx.x & 31) == (__ffs(mask) - 1)) atomicOr(status, 1);
}

__device__ __forceinline__ TurbIn turb_at(const StepArgs& a, int i, int j, int k) {
    TurbIn tb;
    tb.on = false;
    tb.dux = tb.duy = tb.duz = 0.f;
    if (a.uu != nullptr && i == a.iturb) {
        int lit = (*a.d_it) % a.nrturb;
        if (lit == 0) lit = a.nrturb;
        const long long t = (long long)(j - 1) + (long long)a.g.ny * ((long long)(k - 1) + (long long)a.g.nz * lit);
        tb.on = true;
        tb.dux = a.ampl * a.uu[t];
        tb.duy = a.ampl * a.vv[t];
        tb.duz = a.ampl * a.ww[t];
    }
    return tb;
}

// PULL = true : dst(interior) = collide(pull(src))        (steady fused step)
// PULL = false: dst == src, collide in place with rho,u from the arrays in a
//               (the first step after an import, whose moments the caller gave)
template <int Q, typename S, bool PULL>
__global__ void __launch_bounds__(128) k_step(const S* src, S* dst, StepArgs a) {
    const SoaGrid g = a.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > g.nx) return;
    const long long o = g.off(i, j, k);
    const long long rs = g.pitch;
    const long long ps = (long long)g.pitch * (g.ny + 2);

    float fp[Q];
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        const long long d = PULL ? (lat_cx(l) + lat_cy(l) * rs + lat_cz(l) * ps) : 0;
        fp[l] = Store<S>::load(src + (long long)l * g.dstride + o - d);
    }
    const Moments m = moments<Q>(fp);
    float rho, drho, ux, uy, uz;
    if (PULL) {
        drho = m.s0;
        rho = 1.0f + m.s0;
        const float inv = 1.0f / rho;
        ux = m.jx * inv;
        uy = m.jy * inv;
        uz = m.jz * inv;
    } else {
        const long long c = (long long)i + (long long)(g.nx + 2) * ((long long)j + (long long)(g.ny + 2) * k);
        rho = a.rho_in[c];
        drho = rho - 1.0f;
        ux = a.u_in[c];
        uy = a.v_in[c];
        uz = a.w_in[c];
    }
    flag_bad_density(a.status, rho, ux, uy, uz);
    const bool solid = a.solid ? a.solid[((long long)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1)] != 0 : false;
    const float abl = a.abl ? a.abl[k - 1] : 0.0f;
    const TurbIn tb = turb_at(a, i, j, k);
    collide<Q>(fp, m, drho, rho, ux, uy, uz, a.cp, abl, a.cp.tau0, solid, tb);
#pragma unroll
    for (int l = 0; l < Q; ++l) Store<S>::store(dst + (long long)l * g.dstride + o, fp[l]);
}

// Advance the device step counter after the boundary kernels of a step.
__global__ void k_bump_step(int* d_it) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *d_it += 1;
}

// Reference layout (absolute FP32) -> state (offsets in S).  One block per
// (row, chunk of 128 cells); the row is staged through shared memory so both
// the strided reference reads and the per-direction writes are coalesced.
template <int Q, typename S>
__global__ void __launch_bounds__(128) k_import(const float* __restrict__ ref, S* __restrict__ dst, SoaGrid g) {
    __shared__ float sm[128 * Q];
    const int i0 = blockIdx.x * 128;
    const int j = blockIdx.y, k = blockIdx.z;
    const int n = min(128, g.nx + 2 - i0);
    if (n <= 0) return;
    const long long base = ((long long)i0 + (long long)(g.nx + 2) * ((long long)j + (long long)(g.ny + 2) * k)) * Q;
    for (int e = threadIdx.x; e < n * Q; e += blockDim.x) sm[e] = ref[base + e];
    __syncthreads();
    const int t = threadIdx.x;
    if (t < n) {
        const long long o = g.off(i0 + t, j, k);
#pragma unroll
        for (int l = 0; l < Q; ++l) dst[(long long)l * g.dstride + o] = Store<S>::from_f(sm[t * Q + l] - lat_w<Q>(l));
    }
}

// State -> reference layout.  PULL: interior cells take the streamed values
// pulled from `src` (the reference's f1 after drift), ghost cells are copied
// from `ghost`.  Otherwise every cell is copied from `src`.
template <int Q, typename S, bool PULL>
__global__ void __launch_bounds__(128) k_export(const S* __restrict__ src, const S* __restrict__ ghost,
                                                float* __restrict__ ref, SoaGrid g) {
    __shared__ float sm[128 * Q];
    const int i0 = blockIdx.x * 128;
    const int j = blockIdx.y, k = blockIdx.z;
    const int n = min(128, g.nx + 2 - i0);
    if (n <= 0) return;
    const int t = threadIdx.x;
    if (t < n) {
        const int i = i0 + t;
        const bool interior = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
        const long long o = g.off(i, j, k);
        const long long rs = g.pitch, ps = (long long)g.pitch * (g.ny + 2);
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            float v;
            if (PULL && interior) {
                const long long d = lat_cx(l) + lat_cy(l) * rs + lat_cz(l) * ps;
                v = Store<S>::to_f(src[(long long)l * g.dstride + o - d]);
            } else {
                v = Store<S>::to_f((PULL ? ghost : src)[(long long)l * g.dstride + o]);
            }
            sm[t * Q + l] = v + lat_w<Q>(l);
        }
    }
    __syncthreads();
    const long long base = ((long long)i0 + (long long)(g.nx + 2) * ((long long)j + (long long)(g.ny + 2) * k)) * Q;
    for (int e = threadIdx.x; e < n * Q; e += blockDim.x) ref[base + e] = sm[e];
}

// macrovars of the reference's f1 without materialising it: interior cells
// from the pulled values of `src`, ghost cells from `ghost` itself.
template <int Q, typename S>
__global__ void __launch_bounds__(128) k_macro(const S* __restrict__ src, const S* __restrict__ ghost, float* rho,
                                               float* u, float* v, float* w, SoaGrid g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i > g.nx + 1) return;
    const bool interior = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
    const long long o = g.off(i, j, k);
    const long long rs = g.pitch, ps = (long long)g.pitch * (g.ny + 2);
    float fp[Q];
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        const long long d = interior ? (lat_cx(l) + lat_cy(l) * rs + lat_cz(l) * ps) : 0;
        fp[l] = Store<S>::to_f((interior ? src : ghost)[(long long)l * g.dstride + o - d]);
    }
    const Moments m = moments<Q>(fp);
    const float r = 1.0f + m.s0;
    const float inv = 1.0f / r;
    const long long c = (long long)i + (long long)(g.nx + 2) * ((long long)j + (long long)(g.ny + 2) * k);
    rho[c] = r;
    u[c] = m.jx * inv;
    v[c] = m.jy * inv;
    w[c] = m.jz * inv;
}

}  // namespace lbm
