// tma_step.cuh -- the steady fused step with TMA-staged shared-memory tiles.
//
// Same update as k_step_fast (state_kernels.cuh), but the pulled populations
// reach the threads through shared memory: for every tile of 128 cells along
// i of one row (j,k), one warp issues Q bulk copies (cp.async.bulk, the 1-D
// TMA path) of the source row segments (i0-4 .. i0+131 for FP32) of each
// direction into a pipeline stage, completing on an mbarrier.  A CTA walks its
// tiles with NST stages in flight, so the bytes in flight per SM no longer
// depend on registers, and each thread reads its Q values from shared memory
// at fixed offsets instead of forming Q global addresses.
//
// Waits are bounded: a stage that does not complete within the iteration limit
// sets LBM_STATUS_TIMEOUT and the CTA stops.  Every copy lands in the issuing CTA's own shared memory only.
#pragma once

#include "state_kernels.cuh"

namespace lbm {

enum { LBM_STATUS_TIMEOUT_BIT = 2 };

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// 1-D bulk copy global -> this CTA's shared memory, completing on bar (this CTA only)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Segment of one direction's source row per tile: FP32 i0-4 .. i0+131 (136
// elements, 544 B), FP16 i0-8 .. i0+135 (144 elements, 288 B); both start on a
// 16-byte boundary because interior i=1 sits on a 128-byte boundary.
template <typename S>
struct Seg {
    static constexpr int lead = sizeof(S) == 4 ? 4 : 8;
    static constexpr int elems = sizeof(S) == 4 ? 136 : 144;
    static constexpr int bytes = elems * (int)sizeof(S);
};

constexpr int kTmaStages = 3;
constexpr int kTileCells = 128;
constexpr long long kTmaSpinLimit = 1LL << 24;

template <int Q, typename S>
__host__ __device__ constexpr int tma_smem_bytes() {
    return kTmaStages * Q * Seg<S>::bytes + 128;
}

// Issue the Q segment copies of tile t into stage buffer st (called by warp 0).
template <int Q, typename S, bool WRAP>
__device__ __forceinline__ void tma_issue(const S* src, const StepArgs& a, long long t, int nbx, unsigned char* st,
                                          uint64_t* bar) {
    const SoaGrid& g = a.g;
    const int b = (int)(t % nbx);
    const long long jk = t / nbx;
    const int j = (int)(jk % g.ny) + 1;
    const int k = (int)(jk / g.ny) + 1;
    const int i0 = 1 + b * kTileCells;
    const int lane = threadIdx.x & 31;
    if (lane == 0) mbar_expect_tx(bar, (unsigned)(Q * Seg<S>::bytes));
    __syncwarp();
    if (lane < Q) {
        const int l = lane;
        int js = j - c_cy[l];
        if (WRAP) js = wrapj(js, g.ny);
        const int ks = k - c_cz[l];
        const S* gsrc = src + (long long)l * g.dstride + g.off(i0 - Seg<S>::lead, js, ks);
        bulk_load(st + l * Seg<S>::bytes, gsrc, (unsigned)Seg<S>::bytes, bar);
    }
}

template <int Q, typename S, int L>
struct SmemLoad {
    static __device__ __forceinline__ void run(float (&fp)[Q], const S* seg0, int t) {
        const S* p = seg0 + L * Seg<S>::elems + (t + Seg<S>::lead - lat_cx(L));
        if constexpr (sizeof(S) == 2) fp[L] = __half2float(*p);
        else fp[L] = *p;
        SmemLoad<Q, S, L + 1>::run(fp, seg0, t);
    }
};
template <int Q, typename S>
struct SmemLoad<Q, S, Q> {
    static __device__ __forceinline__ void run(float (&)[Q], const S*, int) {}
};

template <int Q, typename S, bool WRAP>
__global__ void __launch_bounds__(128, 4) k_step_tma(const S* __restrict__ src, S* __restrict__ dst, StepArgs a,
                                                     long long ntiles) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
    unsigned char* stages = smem + 128;
    const int nbx = (a.g.nx + kTileCells - 1) / kTileCells;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < kTmaStages; ++s) mbar_init(&bars[s], 1);
        fence_proxy_async_smem();
    }
    __syncthreads();
    // prologue: the first kTmaStages tiles of this CTA
    if (tid < 32) {
        for (int s = 0; s < kTmaStages; ++s) {
            const long long t = blockIdx.x + (long long)s * gridDim.x;
            if (t < ntiles) tma_issue<Q, S, WRAP>(src, a, t, nbx, stages + s * Q * Seg<S>::bytes, &bars[s]);
        }
    }
    int it = 0;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int s = it % kTmaStages;
        const unsigned parity = (unsigned)((it / kTmaStages) & 1);
        long long spin = 0;
        while (!mbar_try_wait(&bars[s], parity)) {
            if (++spin > kTmaSpinLimit) {
                if (tid == 0) atomicOr(a.status, 1 << LBM_STATUS_TIMEOUT_BIT);
                return;
            }
        }
        const S* seg0 = reinterpret_cast<const S*>(stages + s * Q * Seg<S>::bytes);
        float fp[Q];
        SmemLoad<Q, S, 0>::run(fp, seg0, tid);
        __syncthreads();   // every thread has its values: stage s may be refilled
        if (tid < 32) {
            const long long tn = t + (long long)kTmaStages * gridDim.x;
            if (tn < ntiles) {
                if (tid == 0) fence_proxy_async_smem();
                __syncwarp();
                tma_issue<Q, S, WRAP>(src, a, tn, nbx, stages + s * Q * Seg<S>::bytes, &bars[s]);
            }
        }
        const int b = (int)(t % nbx);
        const long long jk = t / nbx;
        const int j = (int)(jk % a.g.ny) + 1;
        const int k = (int)(jk / a.g.ny) + 1;
        const int i = 1 + b * kTileCells + tid;
        if (i <= a.g.nx) cell_update<Q, S, WRAP>(fp, dst, a, i, j, k);
    }
}

}  // namespace lbm
