// ensemble.cuh -- one launch per phase for a whole ensemble of independent runs.
//
// An ensemble is a set of members of different sizes, each a complete fused
// state (its own buffers, boundaries, inflow, turbulence fields and step
// counter) in the folded configuration.  The step of every member runs in one
// launch of k_ens_step and the boundaries of every member in one launch of
// k_ens_bc.  The blocks of a launch are dealt out member by member, so a block
// never straddles two members.  A block reads its (member, block within the
// member) from a per-launch table (one load, no search), copies that member's
// StepArgs into shared memory and then runs the same
// per-pair (pair_cell) or per-block (bc_fold_block) code as the single-state
// kernels, so a member of an ensemble computes exactly what it computes alone.
//
// In k_ens_step a block of T threads covers R consecutive tiles of T
// consecutive pairs of the member's pairs flattened row by row (pair q:
// i = 2 (q mod nx/2) + 1, row q div nx/2), so rows shorter than a block leave
// no threads idle, and a block's set-up (its table entry and the member's
// arguments) serves R tiles.
#pragma once

#include "pair_step.cuh"

namespace lbm {

struct EnsMember {
    StepArgs a[2];       // arguments of a step whose source is buffer p (p = parity)
    void* buf[2];
    int nface_blocks;    // k_bc_fold layout of this member (blocks of 128 threads)
    FastDiv hp, ny;      // division by the pairs per row (nx / 2) and by ny: the pair decode
};

struct EnsLayout {
    const EnsMember* mem;
    const int2* blk;     // per block of this launch's grid: (member, block index within the member)
};

// the member's arguments into shared memory, in 16-byte words (StepArgs is
// 16-byte aligned: one load per thread for blocks of 64 threads or more)
__device__ __forceinline__ void ens_load_args(unsigned char* raw, const StepArgs* ga) {
    static_assert(sizeof(StepArgs) % 16 == 0, "StepArgs is copied in 16-byte words");
    constexpr int n = (int)(sizeof(StepArgs) / 16);
    for (int w = threadIdx.x; w < n; w += blockDim.x)
        reinterpret_cast<uint4*>(raw)[w] = __ldg(reinterpret_cast<const uint4*>(ga) + w);
    __syncthreads();
}

template <int Q, typename S, int T, int MINB, int R>
__global__ void __launch_bounds__(T, MINB) k_ens_step(EnsLayout L, int parity) {
    __shared__ __align__(16) unsigned char raw[sizeof(StepArgs)];
    const int2 mb = __ldg(L.blk + blockIdx.x);
    const EnsMember* em = L.mem + mb.x;
    ens_load_args(raw, &em->a[parity]);
    const StepArgs& a = *reinterpret_cast<const StepArgs*>(raw);
    // 32-bit decode by multiply-high (a member holds fewer than 2^31 pairs)
    const unsigned hp = (unsigned)(a.g.nx / 2);
    const unsigned npairs = hp * (unsigned)a.g.ny * (unsigned)a.g.nz;
    const S* src = reinterpret_cast<const S*>(em->buf[parity]);
    S* dst = reinterpret_cast<S*>(em->buf[1 - parity]);
    for (int r = 0; r < R; ++r) {
        const unsigned q = ((unsigned)mb.y * R + r) * T + threadIdx.x;
        if (q >= npairs) return;   // the later tiles are past the member's end too
        const unsigned row = fdiv(q, em->hp);
        const int i = 2 * (int)(q - row * hp) + 1;
        const unsigned kk = fdiv(row, em->ny);
        const int j = (int)(row - kk * (unsigned)a.g.ny) + 1;
        const int k = (int)kk + 1;
        pair_cell<Q, S, true>(src, dst, a, i, j, k);
    }
}

template <int Q, typename S>
__global__ void __launch_bounds__(128) k_ens_bc(EnsLayout L, int parity) {
    __shared__ __align__(16) unsigned char raw[sizeof(StepArgs)];
    const int2 mb = __ldg(L.blk + blockIdx.x);
    const EnsMember* em = L.mem + mb.x;
    ens_load_args(raw, &em->a[parity]);
    const StepArgs& a = *reinterpret_cast<const StepArgs*>(raw);
    bc_fold_block<Q, S, true>(reinterpret_cast<S*>(em->buf[1 - parity]), reinterpret_cast<const S*>(em->buf[parity]), a,
                              em->nface_blocks, mb.y);
}

}  // namespace lbm
