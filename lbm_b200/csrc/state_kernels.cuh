// state_kernels.cuh -- kernels of the fused state (structure of arrays).
//
// One launch of k_step performs, for every interior cell, what the reference
// does in drift -> macrovars -> inflow_turbulence_forcing -> postcoll ->
// inflow_turbulence_apply -> solids (main.F90:322-329 of step n-1 and
// :296-310 of step n): it pulls the post-collision populations of the
// neighbours, forms the moments in registers, collides, and writes the new
// post-collision populations once.
//
// Boundaries.  In the general case the ghost kernels of boundary.cuh then run
// in the reference's order.  For the configuration the reference runs
// (inflow/outflow in i, periodic j, closed k: ibnd=1, jbnd=0, kbnd in
// {11,12,21,22}) the step kernel also writes the ghost cells itself ("folded"
// boundaries), reproducing boundarycond (m_boundarycond.F90:108-365) value
// for value, with one extra launch instead of four:
//   * periodic j: the ghost rows j=0 and ny+1 are never stored; every reader
//     wraps the row index instead.  After boundarycond the reference's ghost
//     rows are exact copies of rows ny and 1, so wrapping reads the same data.
//   * closed k and inflow/outflow in one kernel, k_bc_fold, in which the
//     reference's ordering (k-faces read x-ghost columns before the inflow
//     rewrites them) is kept by giving each x-ghost element a single thread
//     that reads its old value and then writes the new one.
//   * x-ghost columns (i = 0 and nx+1): each buffer keeps them whole in a
//     compact array written coalesced by k_bc_fold; the rows hold only the
//     directions a pull reads (cx > 0 at i = 0, cx < 0 at nx+1).
#pragma once

#include "collide_rows.cuh"

namespace lbm {

// n / d for 0 <= n < 2^31 by a multiply-high and a shift (Granlund-Montgomery
// round-up method: m = ceil(2^(31+l) / d), l = ceil(log2 d), shift l - 1); d = 1
// is the identity
struct FastDiv {
    unsigned d, m;
    int s;
};
inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f;
    f.d = d < 1u ? 1u : d;
    int l = 0;
    while ((1ull << l) < f.d) ++l;
    f.m = f.d == 1u ? 0u : (unsigned)(((1ull << (31 + l)) + f.d - 1) / f.d);
    f.s = l > 0 ? l - 1 : 0;
    return f;
}
__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv& f) {
    return f.d == 1u ? n : (__umulhi(n, f.m) >> f.s);
}

// 16-byte aligned: the ensemble kernels copy it into shared memory in 16-byte words
struct alignas(16) StepArgs {
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
    // folded boundaries
    int kopt_lo, kopt_hi;     // -1 no-slip, +1 free-slip at k=1 / k=nz
    const float* uvel;        // inflow profile uvel(nz)
    float rho0, cosd, sind;   // inflow constants (m_boundary_i_inflow_kernel.F90:35,71-73)
    int* d_it_rw;             // step counter, advanced by the boundary kernel
    void* edge;               // post-collision populations at i=1 and i=nx: [side][l][k-1][j-1]
    int full_sector;          // x-ghost sectors hold nothing but the ghost and padding
    void* xg_dst;             // x-ghost columns of the buffer the step writes: [side][l][k-1][j-1]
    const float* force;       // external_forcing(3,0:nx+1,0:ny+1,0:nz+1) or null (pair kernel only)
    // 32-bit element offsets of k_step_fast, computed on the host:
    int poff[27];             // pull source of direction l relative to the cell: l*dstride - (cx + cy*pitch + cz*plane)
    int soff[27];             // l*dstride
    long long poffb[27];      // poff and soff in bytes, for the pair kernel: a 64-bit constant operand
    long long soffb[27];      // per address instead of a sign-extended, scaled 32-bit offset
};

__device__ __forceinline__ void flag_bad_density(int* status, float rho, float ux, float uy, float uz) {
    const float chk = rho + ux + uy + uz;
    const bool bad = !(rho > 0.0f) || !(fabsf(chk) < 1.0e30f);
    const unsigned mask = __activemask();
    const unsigned vote = __ballot_sync(mask, bad);
    if (vote && (threadIdx.x & 31) == (__ffs(mask) - 1)) atomicOr(status, 1);
}

// flag_bad_density for two cells with one vote: rho of both cells and chk = rho + u + v + w of each
__device__ __forceinline__ void flag_bad_density2(int* status, float2 rho, float2 chk) {
    const bool bad = !(rho.x > 0.0f) || !(rho.y > 0.0f) || !(fabsf(chk.x) < 1.0e30f) || !(fabsf(chk.y) < 1.0e30f);
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
        tb.dux = __fmul_rn(a.ampl, a.uu[t]);   // rounded here: never fused into a later add
        tb.duy = __fmul_rn(a.ampl, a.vv[t]);
        tb.duz = __fmul_rn(a.ampl, a.ww[t]);
    }
    return tb;
}

// periodic row index for j in 0..ny+1
__device__ __forceinline__ int wrapj(int j, int ny) { return j == 0 ? ny : (j == ny + 1 ? 1 : j); }

// element distance from cell (i,j,k) back to its pull source (i-cx, j-cy, k-cz);
// with wrap, a source row 0 or ny+1 is replaced by row ny or 1 (j interior)
template <int L>
__device__ __forceinline__ long long pull_delta(const SoaGrid& g, int j, bool wrap) {
    const long long rs = g.pitch, ps = (long long)g.pitch * (g.ny + 2);
    long long d = lat_cx(L) + lat_cy(L) * rs + lat_cz(L) * ps;
    if (wrap) {
        if (lat_cy(L) > 0 && j == 1) d -= (long long)g.ny * rs;
        if (lat_cy(L) < 0 && j == g.ny) d += (long long)g.ny * rs;
    }
    return d;
}

template <int Q, typename S, int L>
struct PullLoop {
    static __device__ __forceinline__ void run(float (&fp)[Q], const S* src, const SoaGrid& g, long long o, int j,
                                               bool wrap) {
        fp[L] = Store<S>::load(src + (long long)L * g.dstride + o - pull_delta<L>(g, j, wrap));
        PullLoop<Q, S, L + 1>::run(fp, src, g, o, j, wrap);
    }
};
template <int Q, typename S>
struct PullLoop<Q, S, Q> {
    static __device__ __forceinline__ void run(float (&)[Q], const S*, const SoaGrid&, long long, int, bool) {}
};

// Folded configuration: index of ghost (side ? nx+1 : 0, j, k), direction l, in
// a buffer's compact x-ghost array xg[side][l][k-1][j-1] (j, k interior).
__device__ __forceinline__ long long xg_index(const SoaGrid& g, int Q, int side, int l, int j, int k) {
    return ((long long)(side * Q + l) * g.nz + (k - 1)) * g.ny + (j - 1);
}

// Store one 32-byte sector (two 16-byte vectors) holding v at element `slot`
// and zeros elsewhere; p is 32-byte aligned.
template <typename S>
__device__ __forceinline__ void store_sector(S* p, S v, int slot) {
    unsigned int w[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
    if (sizeof(S) == 4) {
        w[slot] = *reinterpret_cast<const unsigned int*>(&v);
    } else {
        const unsigned int h = *reinterpret_cast<const unsigned short*>(&v);
        w[slot >> 1] = (slot & 1) ? (h << 16) : h;
    }
    uint4* q = reinterpret_cast<uint4*>(p);
    q[0] = make_uint4(w[0], w[1], w[2], w[3]);
    q[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

// The inflow ghost value of a direction whose source is the post-collision
// value fin of direction ls (weight wl, velocity (cx, cy)) at the cell i = 1,
// with uu the inflow speed of the cell's k
// (m_boundary_i_inflow_kernel.F90:56-111): fin - 2 wl rho0 (cx uu cos + cy uu
// sin) / cs2, rounded operation by operation in that order.
__device__ __forceinline__ float inflow_value(float fin, float wl, int cx, int cy, float uu, const StepArgs& a) {
    const float t = __fadd_rn(__fmul_rn(__fmul_rn((float)cx, uu), a.cosd), __fmul_rn(__fmul_rn((float)cy, uu), a.sind));
    const float p = __fmul_rn(__fmul_rn(__fmul_rn(2.0f, wl), a.rho0), t);
    return __fsub_rn(fin, __fdiv_rn(p, 1.0f / 3.0f));
}

// Boundary kernel of the folded configuration, run after k_step on the new
// buffer f1 (= dst of the step) with f2 the old buffer.  Two kinds of threads,
// each issuing all its loads before its first store (the stores go to ghost
// cells none of its loads reads, but the compiler cannot prove it), so that a
// thread waits on memory once:
//   * k-face threads, one per (i, j, face) with i in 1..nx: for each outgoing
//     direction l of the face, f1(l,i,j,kg) = f1(l, i-cx, j-cy, kp) when the
//     source is an interior cell, and f1(m,i,j,kg) = f2(l,i,j,kg) for the
//     reflected direction m (m_boundary_k_closed_kernel.F90:35-46).
//   * x-ghost threads: the inflow ghost (0,j,k) and the outflow ghost
//     (nx+1,j,k) (m_boundary_i_inflow_kernel.F90:56-111), written to the
//     compact x-ghost array, and into the rows for the directions the next pull
//     reads there (cx > 0 at i = 0, cx < 0 at nx+1).  At the planes k=1 and
//     k=nz they first pass the value those row ghosts held before this step to
//     the k-ghost cell that the reference's k-face copies it to (1 or nx, j+cy,
//     kg), so each ghost is read and then written by one and the same thread.
//     WIDE: one thread per (j, k, side) with every direction (fewer, longer
//     threads: faster for the short columns of small ensemble members); else
//     one thread per (j, l, k), both sides (faster for large domains).
// vb: this block's index among the nface_blocks + x-ghost blocks of the grid
// (blocks of 128 threads).
template <int Q, typename S, int SIDE>
__device__ __forceinline__ void bc_fold_face(S* f1, const S* f2, const SoaGrid& g, int opt, int i, int j) {
    constexpr int NO = (Q == 27) ? 9 : 5;   // outgoing directions of a face
    const int kp = SIDE ? g.nz : 1, kg = SIDE ? g.nz + 1 : 0;
    const long long og = g.off(i, j, kg);
    S cp[NO], rf[NO];
    bool in[NO];
    int n = 0;
#pragma unroll
    for (int l = 1; l < Q; ++l) {
        const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
        if (SIDE ? (cz <= 0) : (cz >= 0)) continue;
        const int si = i - cx;
        in[n] = si >= 1 && si <= g.nx;
        if (in[n]) cp[n] = f1[(long long)l * g.dstride + g.off(si, wrapj(j - cy, g.ny), kp)];
        rf[n] = f2[(long long)l * g.dstride + og];
        ++n;
    }
    n = 0;
#pragma unroll
    for (int l = 1; l < Q; ++l) {
        const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
        if (SIDE ? (cz <= 0) : (cz >= 0)) continue;
        if (in[n]) f1[(long long)l * g.dstride + og] = cp[n];
        const int m = opt < 0 ? lat_opposite(l) : lat_find<Q>(cx, cy, -cz);
        f1[(long long)m * g.dstride + og] = rf[n];
        ++n;
    }
}

template <int Q, typename S, int SIDE>
__device__ __forceinline__ void bc_fold_xcol(S* f1, const StepArgs& a, int j, int k, long long cell) {
    const SoaGrid& g = a.g;
    const long long nyz = (long long)g.ny * g.nz;
    const S* edge = (const S*)a.edge + (long long)SIDE * Q * nyz + cell;   // cell 1 (side 0) or nx (side 1)
    S* xg = (S*)a.xg_dst + (long long)SIDE * Q * nyz + cell;                 // xg_index(g, Q, SIDE, l, j, k)
    const int ig = SIDE ? g.nx + 1 : 0;   // the ghost column
    S ev[Q];
#pragma unroll
    for (int l = 0; l < Q; ++l) ev[l] = edge[l * nyz];
    const float uu = SIDE ? 0.0f : a.uvel[k - 1];
    if (k == 1 || k == g.nz) {
        constexpr int NS = (Q == 27) ? 9 : 5;   // directions the pull reads at this ghost
        const int kg = (k == 1) ? 0 : g.nz + 1;
        const int ib = SIDE ? g.nx : 1;
        S old[NS];
        int n = 0;
#pragma unroll
        for (int l = 1; l < Q; ++l) {
            if (SIDE ? (lat_cx(l) >= 0) : (lat_cx(l) <= 0)) continue;
            old[n++] = f1[(long long)l * g.dstride + g.off(ig, j, k)];
        }
        n = 0;
#pragma unroll
        for (int l = 1; l < Q; ++l) {
            const int cy = lat_cy(l), cz = lat_cz(l);
            if (SIDE ? (lat_cx(l) >= 0) : (lat_cx(l) <= 0)) continue;
            if ((k == 1) ? (cz < 0) : (cz > 0)) f1[(long long)l * g.dstride + g.off(ib, wrapj(j + cy, g.ny), kg)] = old[n];
            ++n;
        }
    }
    constexpr int spe = 32 / (int)sizeof(S);
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        S v;
        if (SIDE == 0) {
            // directions with cx > 0 take the corrected value of their opposite
            const int ls = lat_cx(l) > 0 ? lat_opposite(l) : l;
            v = Store<S>::from_f(inflow_value(Store<S>::to_f(ev[ls]), lat_w<Q>(ls), lat_cx(ls), lat_cy(ls), uu, a));
        } else {
            v = ev[l];   // zero gradient
        }
        xg[l * nyz] = v;
        // the rows: a ghost's 32-byte sector holds nothing else but row padding, so
        // it is written whole (no read-modify-write of a partial sector)
        if (SIDE ? (lat_cx(l) < 0) : (lat_cx(l) > 0)) {
            S* p = f1 + (long long)l * g.dstride + g.off(ig, j, k);
            if (a.full_sector) store_sector<S>(SIDE ? p : p - (spe - 1), v, SIDE ? 0 : spe - 1);
            else *p = v;
        }
    }
}

// one x-ghost thread per (j, l, k), both sides (j fastest, packed: no idle
// threads for short rows; 32-bit index arithmetic up to 2^31 elements)
template <int Q, typename S>
__device__ __forceinline__ void bc_fold_xelem(S* f1, const StepArgs& a, long long e) {
    const SoaGrid& g = a.g;
    const long long nyz = (long long)g.ny * g.nz;
    const long long ne = (long long)Q * nyz;
    int j, l, k;
    if (ne < (1LL << 31)) {
        const unsigned ue = (unsigned)e, uny = (unsigned)g.ny;
        const unsigned r = ue / uny;
        j = (int)(ue - r * uny) + 1;
        l = (int)(r % (unsigned)Q);
        k = (int)(r / (unsigned)Q) + 1;
    } else {
        j = (int)(e % g.ny) + 1;
        l = (int)((e / g.ny) % Q);
        k = (int)(e / ((long long)g.ny * Q)) + 1;
    }
    const int cx = c_cx[l], cy = c_cy[l], cz = c_cz[l];
    S* fl = f1 + (long long)l * g.dstride;
    if (k == 1 || k == g.nz) {
        const bool out = (k == 1) ? (cz < 0) : (cz > 0);
        if (out) {
            const int kg = (k == 1) ? 0 : g.nz + 1;
            if (cx > 0) fl[g.off(1, wrapj(j + cy, g.ny), kg)] = fl[g.off(0, j, k)];
            if (cx < 0) fl[g.off(g.nx, wrapj(j + cy, g.ny), kg)] = fl[g.off(g.nx + 1, j, k)];
        }
    }
    const S* edge = (const S*)a.edge;
    const long long cell = (long long)(k - 1) * g.ny + (j - 1);
    // inflow: directions with cx > 0 take the corrected value of their opposite
    const int ls = (cx > 0) ? c_opp[l] : l;
    const float fin = Store<S>::to_f(edge[(long long)ls * nyz + cell]);
    const S gin = Store<S>::from_f(inflow_value(fin, c_w[Q == 27 ? 1 : 0][ls], c_cx[ls], c_cy[ls], a.uvel[k - 1], a));
    // outflow: zero gradient
    const S gout = edge[((long long)Q + l) * nyz + cell];
    S* xg = (S*)a.xg_dst;
    xg[xg_index(g, Q, 0, l, j, k)] = gin;
    xg[xg_index(g, Q, 1, l, j, k)] = gout;
    constexpr int spe = 32 / (int)sizeof(S);
    if (cx > 0) {
        S* p = fl + g.off(0, j, k);
        if (a.full_sector) store_sector<S>(p - (spe - 1), gin, spe - 1);
        else *p = gin;
    }
    if (cx < 0) {
        S* p = fl + g.off(g.nx + 1, j, k);
        if (a.full_sector) store_sector<S>(p, gout, 0);
        else *p = gout;
    }
}

template <int Q, typename S, bool WIDE>
__device__ __forceinline__ void bc_fold_block(S* f1, const S* f2, const StepArgs& a, int nface_blocks, int vb) {
    const SoaGrid& g = a.g;
    if (vb < nface_blocks) {
        int side, i, j;
        if (WIDE) {
            // (i, j, face) flattened, i fastest: no idle threads for rows shorter than a block
            const long long e = (long long)vb * 128 + threadIdx.x;
            const long long nxy = (long long)g.nx * g.ny;
            if (e >= 2 * nxy) return;
            side = e >= nxy ? 1 : 0;
            const long long r = e - side * nxy;
            j = (int)(r / g.nx) + 1;
            i = (int)(r - (long long)(j - 1) * g.nx) + 1;
        } else {
            const int per_row = (g.nx + 127) / 128;
            const int b = vb;
            side = b / (per_row * g.ny);
            j = (b / per_row) % g.ny + 1;
            i = (b % per_row) * 128 + threadIdx.x + 1;
            if (i > g.nx) return;
        }
        if (side) bc_fold_face<Q, S, 1>(f1, f2, g, a.kopt_hi, i, j);
        else bc_fold_face<Q, S, 0>(f1, f2, g, a.kopt_lo, i, j);
        return;
    }
    const long long nyz = (long long)g.ny * g.nz;
    const long long e = (long long)(vb - nface_blocks) * 128 + threadIdx.x;
    if (e >= (WIDE ? 2 : Q) * nyz) return;
    if (e == 0) *a.d_it_rw += 1;   // the step counter advances once per step
    if (!WIDE) {
        bc_fold_xelem<Q, S>(f1, a, e);
        return;
    }
    // side 0 for every (j, k), then side 1, j fastest
    const int side = e >= nyz ? 1 : 0;
    const long long cell = e - side * nyz;
    const int j = (int)(cell % g.ny) + 1;
    const int k = (int)(cell / g.ny) + 1;
    if (side) bc_fold_xcol<Q, S, 1>(f1, a, j, k, cell);
    else bc_fold_xcol<Q, S, 0>(f1, a, j, k, cell);
}

// blocks of bc_fold_block: the k-face blocks, then the x-ghost blocks (WIDE:
// the ensemble's layout, k-face threads flattened over (i, j, face))
__host__ __device__ inline int bc_fold_face_blocks(const SoaGrid& g, bool wide = false) {
    return wide ? (int)((2LL * g.nx * g.ny + 127) / 128) : 2 * g.ny * ((g.nx + 127) / 128);
}
__host__ __device__ inline long long bc_fold_xg_blocks(const SoaGrid& g, int Q, bool wide) {
    return ((wide ? 2LL : (long long)Q) * g.ny * g.nz + 127) / 128;
}


template <int Q, typename S>
__global__ void __launch_bounds__(128) k_bc_fold(S* f1, const S* f2, StepArgs a, int nface_blocks) {
    pdl_enter();
    bc_fold_block<Q, S, false>(f1, f2, a, nface_blocks, blockIdx.x);
}

// The ghost cells of a state buffer, numbered t = 0 .. ghost_cells(g) - 1: whole
// rows with k in {0, nz+1} or j in {0, ny+1}, then i in {0, nx+1} of the other
// rows.  Returns false past the last one.
__device__ __forceinline__ bool ghost_cell(const SoaGrid& g, long long t, int& i, int& j, int& k) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long nfull = (2LL * (ny + 2) + 2LL * nz) * (nx + 2);
    if (t < nfull) {
        const long long r = t / (nx + 2);
        i = (int)(t - r * (nx + 2));
        if (r < 2LL * (ny + 2)) {
            k = (r < ny + 2) ? 0 : nz + 1;
            j = (int)(r % (ny + 2));
        } else {
            const int q = (int)(r - 2LL * (ny + 2));
            j = (q < nz) ? 0 : ny + 1;
            k = 1 + q % nz;
        }
        return true;
    }
    const long long u = t - nfull;
    if (u >= 2LL * ny * nz) return false;
    i = (u & 1) ? nx + 1 : 0;
    const long long r = u >> 1;
    j = 1 + (int)(r % ny);
    k = 1 + (int)(r / ny);
    return true;
}
inline long long ghost_cells(const SoaGrid& g) {
    return (2LL * (g.ny + 2) + 2LL * g.nz) * (g.nx + 2) + 2LL * g.ny * g.nz;
}

// Copy every ghost entry (all directions) of one state buffer to another: the
// ghost cells a step leaves alone, or fills from the buffer's own earlier
// contents (the two-timestep bounce-back), as the buffer it replaces held them.
// A thread per ghost cell, blockIdx.y = direction.
template <typename T>
__global__ void __launch_bounds__(128) k_copy_ghosts(T* __restrict__ dst, const T* __restrict__ src, SoaGrid g) {
    int i, j, k;
    if (!ghost_cell(g, (long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
    const long long o = (long long)blockIdx.y * g.dstride + g.off(i, j, k);
    dst[o] = src[o];
}

// k_copy_ghosts for the folded configuration, which reads fewer ghost entries of
// a buffer: the k ghost rows (j = 1..ny, every i; exports read them whole) and the
// x ghosts of the rows k = 1 and nz (the boundary kernel reads them two steps
// after they were written).  The other x ghosts are rewritten by every step where
// a step reads them and exported from the compact x-ghost arrays, and periodic j
// rows are read as rows ny and 1.  A thread per cell, blockIdx.y = direction.
template <typename T>
__global__ void __launch_bounds__(128) k_copy_ghosts_fold(T* __restrict__ dst, const T* __restrict__ src, SoaGrid g) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long nrow = 2LL * ny * (nx + 2);
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (t < nrow) {
        const long long r = t / (nx + 2);
        i = (int)(t - r * (nx + 2));
        j = 1 + (int)(r % ny);
        k = (r < ny) ? 0 : nz + 1;
    } else {
        const long long u = t - nrow;
        const int nk = (nz > 1) ? 2 : 1;
        if (u >= 2LL * nk * ny) return;
        i = (u & 1) ? nx + 1 : 0;
        const long long r = u >> 1;
        j = 1 + (int)(r % ny);
        k = (r < ny) ? 1 : nz;
    }
    const long long o = (long long)blockIdx.y * g.dstride + g.off(i, j, k);
    dst[o] = src[o];
}
inline long long fold_ghost_cells(const SoaGrid& g) {
    return 2LL * g.ny * (g.nx + 2) + 2LL * ((g.nz > 1) ? 2 : 1) * g.ny;
}

// Plane j of a state buffer (every i = 0..nx+1, k = 0..nz+1 and direction) to or
// from a contiguous array buf[l][k][i]: the halo planes of a j slab.  UNPACK:
// buf -> buffer.  xg (packing, folded configuration): the compact x-ghost array
// of the buffer, which holds every direction of the x ghosts of rows 1..ny (the
// rows hold only the pulled ones).  One thread per element of buf, flat (the
// plane is 2 KB row segments spread over the whole buffer; more elements per
// thread measured no faster).
template <typename T, bool UNPACK>
__global__ void __launch_bounds__(256) k_halo_plane(T* buf, T* f, SoaGrid g, int j, int Q, const T* __restrict__ xg) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int w = g.nx + 2;
    const long long n = (long long)Q * (g.nz + 2) * w;
    if (q >= n) return;
    const long long r = q / w;
    const int i = (int)(q - r * w);
    const int k = (int)(r % (g.nz + 2)), l = (int)(r / (g.nz + 2));
    const long long o = (long long)l * g.dstride + g.off(i, j, k);
    if (UNPACK) {
        f[o] = buf[q];
    } else {
        const bool fromxg = xg && (i == 0 || i == g.nx + 1) && k >= 1 && k <= g.nz && j >= 1 && j <= g.ny;
        buf[q] = fromxg ? xg[xg_index(g, Q, i == 0 ? 0 : 1, l, j, k)] : f[o];
    }
}

// The ghost shell of a state buffer to or from a compact array
// packed[l][t] (t: ghost_cell numbering).  UNPACK: packed -> buffer.
template <typename T, bool UNPACK>
__global__ void __launch_bounds__(128) k_pack_ghosts(T* packed, T* buf, SoaGrid g, long long ncells) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!ghost_cell(g, t, i, j, k)) return;
    const long long o = (long long)blockIdx.y * g.dstride + g.off(i, j, k);
    const long long q = (long long)blockIdx.y * ncells + t;
    if (UNPACK) buf[o] = packed[q];
    else packed[q] = buf[o];
}

// Folded configuration: copy the x-ghost columns of a buffer whose rows hold
// every direction (after an import or a step with the general boundary
// kernels) into its compact array.  One thread per element of xg.
template <int Q, typename S>
__global__ void __launch_bounds__(128) k_gather_xg(const S* __restrict__ f, S* __restrict__ xg, SoaGrid g) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = 2LL * Q * g.ny * g.nz;
    if (e >= n) return;
    const int j = (int)(e % g.ny) + 1;
    const int k = (int)((e / g.ny) % g.nz) + 1;
    const int l = (int)((e / ((long long)g.ny * g.nz)) % Q);
    const int side = (int)(e / ((long long)g.ny * g.nz * Q));
    xg[e] = f[(long long)l * g.dstride + g.off(side ? g.nx + 1 : 0, j, k)];
}

// PULL = true : dst(interior) = collide(pull(src))        (steady fused step)
// PULL = false: dst == src, collide in place with rho,u from the arrays in a
//               (the first step after an import, whose moments the caller gave)
// WRAP = true : folded configuration: periodic j without stored ghost rows, and
//               the populations at i=1 and i=nx copied to the edge array
template <int Q, typename S, bool PULL, bool WRAP>
__global__ void __launch_bounds__(128, 8) k_step(const S* src, S* dst, StepArgs a) {
    const SoaGrid g = a.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > g.nx) return;
    const long long o = g.off(i, j, k);

    float fp[Q];
    if (PULL) {
        PullLoop<Q, S, 0>::run(fp, src, g, o, j, WRAP);
    } else {
#pragma unroll
        for (int l = 0; l < Q; ++l) fp[l] = Store<S>::load(src + (long long)l * g.dstride + o);
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
    if (WRAP && (i == 1 || i == g.nx)) {
        // the boundary kernel builds the inflow/outflow ghosts from these, read coalesced
        const long long nyz = (long long)g.ny * g.nz;
        S* e = (S*)a.edge + (i == 1 ? 0 : (long long)Q * nyz) + (long long)(k - 1) * g.ny + (j - 1);
#pragma unroll
        for (int l = 0; l < Q; ++l) e[l * nyz] = Store<S>::from_f(fp[l]);
    }
}

// Pull loads of k_step_fast: direction L reads base + poff[L]; sources in row
// j-1 (cy = +1) and j+1 (cy = -1) use bases shifted to the wrapped row.
template <int Q, typename S, int L>
struct Load32 {
    static __device__ __forceinline__ void run(float (&fp)[Q], const S* p0, const S* pyp, const S* pym,
                                               const StepArgs& a) {
        const S* b = lat_cy(L) > 0 ? pyp : (lat_cy(L) < 0 ? pym : p0);
        if constexpr (sizeof(S) == 2) fp[L] = __half2float(__ldg(b + a.poff[L]));   // 2^8-scaled
        else fp[L] = __ldg(b + a.poff[L]);
        Load32<Q, S, L + 1>::run(fp, p0, pyp, pym, a);
    }
};
template <int Q, typename S>
struct Load32<Q, S, Q> {
    static __device__ __forceinline__ void run(float (&)[Q], const S*, const S*, const S*, const StepArgs&) {}
};

// Everything after the loads of one cell of the steady step: moments, collision
// (regularized rows or the plain BGK of collide.cuh), turbulence slice, solid
// swap, stores, and the edge copy of the folded boundaries.  fp holds the pulled
// offsets (2^8-scaled for FP16).
template <int Q, typename S, bool WRAP>
__device__ __forceinline__ void cell_update(float (&fp)[Q], S* __restrict__ dst, const StepArgs& a, int i, int j,
                                            int k) {
    Moments m = moments_rows<Q>(fp);
    constexpr float inv_scale = 1.0f / store_scale<S>();
    if constexpr (sizeof(S) == 2) {
        m.s0 *= inv_scale; m.jx *= inv_scale; m.jy *= inv_scale; m.jz *= inv_scale;
        m.pxx *= inv_scale; m.pyy *= inv_scale; m.pzz *= inv_scale;
        m.pxy *= inv_scale; m.pxz *= inv_scale; m.pyz *= inv_scale;
    }
    const float drho = m.s0;
    const float rho = 1.0f + m.s0;
    const float inv = __frcp_rn(rho);
    const float ux = m.jx * inv, uy = m.jy * inv, uz = m.jz * inv;
    flag_bad_density(a.status, rho, ux, uy, uz);
    const bool solid = a.solid ? a.solid[((long long)(k - 1) * a.g.ny + (j - 1)) * a.g.nx + (i - 1)] != 0 : false;
    const float abl = a.abl ? a.abl[k - 1] : 0.0f;
    if (a.cp.ihrr) {
        collide_rows<Q, S>(fp, m, drho, rho, ux, uy, uz, a.cp, abl, solid);
        if (a.uu != nullptr && i == a.iturb) {
            const TurbIn tb = turb_at(a, i, j, k);
            add_turbulence<Q>(fp, rho, ux, uy, uz, tb, a.cp.ibgk == 3, solid, store_scale<S>());
        }
    } else {
        // plain BGK on the unregularized non-equilibrium (collide.cuh)
#pragma unroll
        for (int l = 0; l < Q; ++l) fp[l] *= inv_scale;
        const TurbIn tb = turb_at(a, i, j, k);
        collide<Q>(fp, m, drho, rho, ux, uy, uz, a.cp, abl, a.cp.tau0, solid, tb);
#pragma unroll
        for (int l = 0; l < Q; ++l) fp[l] *= store_scale<S>();
    }
    S* q = dst + a.g.off(i, j, k);
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        if constexpr (sizeof(S) == 2) q[a.soff[l]] = __float2half_rn(fp[l]);
        else q[a.soff[l]] = fp[l];
    }
    if (WRAP && (i == 1 || i == a.g.nx)) {
        // the boundary kernel builds the inflow/outflow ghosts from these, read coalesced
        const long long nyz = (long long)a.g.ny * a.g.nz;
        S* e = (S*)a.edge + (i == 1 ? 0 : (long long)Q * nyz) + (long long)(k - 1) * a.g.ny + (j - 1);
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            if constexpr (sizeof(S) == 2) e[l * nyz] = __float2half_rn(fp[l]);
            else e[l * nyz] = fp[l];
        }
    }
}

// Steady fused step with the row-organised collision (collide_rows.cuh).  FP16
// state is used in its 2^8-scaled form: the moments are rescaled once and the
// emission constants carry the scale, so no population is multiplied on the way
// in or out.  Needs Q * dstride < 2^31 (32-bit element offsets).
template <int Q, typename S, bool WRAP>
__global__ void __launch_bounds__(128, 8) k_step_fast(const S* __restrict__ src, S* __restrict__ dst, StepArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > a.g.nx) return;
    const long long o = a.g.off(i, j, k);
    float fp[Q];
    {
        const S* p0 = src + o;
        const long long wrapd = (long long)a.g.ny * a.g.pitch;
        const S* pyp = (WRAP && j == 1) ? p0 + wrapd : p0;         // row 0 -> row ny
        const S* pym = (WRAP && j == a.g.ny) ? p0 - wrapd : p0;    // row ny+1 -> row 1
        Load32<Q, S, 0>::run(fp, p0, pyp, pym, a);
    }
    cell_update<Q, S, WRAP>(fp, dst, a, i, j, k);
}

// External forcing of the first step after an import, which collides in place
// with the imported moments (k_step<Q,S,false,...>): adds feq2(rho, u - F/rho) -
// feq2(rho, u) (m_forcings_apply_kernel.F90:47-213) with those moments.  The
// solid swap already ran, so at solid cells the increment's odd part flips.
template <int Q, typename S>
__global__ void __launch_bounds__(128) k_force_state(S* f, StepArgs a) {
    const SoaGrid g = a.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > g.nx) return;
    const long long c = (long long)i + (long long)(g.nx + 2) * ((long long)j + (long long)(g.ny + 2) * k);
    const float rr = a.rho_in[c];
    if (!(rr > 0.0f)) return;
    const float ux = a.u_in[c], uy = a.v_in[c], uz = a.w_in[c];
    const float dux = -a.force[3 * c] / rr, duy = -a.force[3 * c + 1] / rr, duz = -a.force[3 * c + 2] / rr;
    const float dusq = dux * (2.0f * ux + dux) + duy * (2.0f * uy + duy) + duz * (2.0f * uz + duz);
    const bool solid = a.solid ? a.solid[((long long)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1)] != 0 : false;
    const long long o = g.off(i, j, k);
    S* p0 = f + o;
    p0[0] = Store<S>::from_f(Store<S>::to_f(p0[0]) + lat_w<Q>(0) * rr * (-1.5f * dusq));
#pragma unroll
    for (int l = 1; l < Q; l += 2) {
        const int cx = lat_cx(l), cy = lat_cy(l), cz = lat_cz(l);
        const float cu = cdot(cx, cy, cz, ux, uy, uz);
        const float dcu = cdot(cx, cy, cz, dux, duy, duz);
        const float wr = lat_w<Q>(l) * rr;
        const float dE = wr * (4.5f * dcu * (2.0f * cu + dcu) - 1.5f * dusq);
        const float dO = (solid ? -1.0f : 1.0f) * wr * 3.0f * dcu;
        S* pl = f + (long long)l * g.dstride + o;
        S* pm = f + (long long)(l + 1) * g.dstride + o;
        *pl = Store<S>::from_f(Store<S>::to_f(*pl) + dE + dO);
        *pm = Store<S>::from_f(Store<S>::to_f(*pm) + dE - dO);
    }
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
    // eight independent loads in flight per thread before their shared-memory stores
    const int m = n * Q;
    for (int e0 = threadIdx.x; e0 < m; e0 += blockDim.x * 8) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < m) v[u] = ref[base + e];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < m) sm[e] = v[u];
        }
    }
    __syncthreads();
    const int t = threadIdx.x;
    if (t < n) {
        const long long o = g.off(i0 + t, j, k);
#pragma unroll
        for (int l = 0; l < Q; ++l) dst[(long long)l * g.dstride + o] = Store<S>::from_f(sm[t * Q + l] - lat_w<Q>(l));
    }
}

template <int Q, typename S, int L>
struct PullMacro {
    static __device__ __forceinline__ void run(float (&fp)[Q], const S* src, const SoaGrid& g, long long o, int j,
                                               bool wrap) {
        fp[L] = Store<S>::to_f(src[(long long)L * g.dstride + o - pull_delta<L>(g, j, wrap)]);
        PullMacro<Q, S, L + 1>::run(fp, src, g, o, j, wrap);
    }
};
template <int Q, typename S>
struct PullMacro<Q, S, Q> {
    static __device__ __forceinline__ void run(float (&)[Q], const S*, const SoaGrid&, long long, int, bool) {}
};

// State -> reference layout.  PULL: interior cells take the streamed values
// pulled from `src` (the reference's f1 after drift), ghost cells are copied
// from `ghost`.  Otherwise every cell is copied from `src`.  wrap: periodic j,
// ghost rows read from rows ny and 1 (see the file header).  xg: compact
// x-ghost array of the buffer the ghost cells come from, or null.
template <int Q, typename S, bool PULL>
__global__ void __launch_bounds__(128) k_export(const S* __restrict__ src, const S* __restrict__ ghost,
                                                float* __restrict__ ref, SoaGrid g, int wrap,
                                                const S* __restrict__ xg) {
    __shared__ float sm[128 * Q];
    const int i0 = blockIdx.x * 128;
    const int j = blockIdx.y, k = blockIdx.z;
    const int n = min(128, g.nx + 2 - i0);
    if (n <= 0) return;
    const int t = threadIdx.x;
    if (t < n) {
        const int i = i0 + t;
        const bool interior = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
        float v[Q];
        if (PULL && interior) {
            PullMacro<Q, S, 0>::run(v, src, g, g.off(i, j, k), j, wrap != 0);
        } else {
            const int jw = wrap ? wrapj(j, g.ny) : j;
            const long long o = g.off(i, jw, k);
            const S* s = PULL ? ghost : src;
            const bool fromxg = xg && (i == 0 || i == g.nx + 1) && jw >= 1 && jw <= g.ny && k >= 1 && k <= g.nz;
#pragma unroll
            for (int l = 0; l < Q; ++l)
                v[l] = Store<S>::to_f(fromxg ? xg[xg_index(g, Q, i == 0 ? 0 : 1, l, jw, k)] : s[(long long)l * g.dstride + o]);
        }
#pragma unroll
        for (int l = 0; l < Q; ++l) sm[t * Q + l] = v[l] + lat_w<Q>(l);
    }
    __syncthreads();
    const long long base = ((long long)i0 + (long long)(g.nx + 2) * ((long long)j + (long long)(g.ny + 2) * k)) * Q;
    for (int e = threadIdx.x; e < n * Q; e += blockDim.x) ref[base + e] = sm[e];
}

// macrovars of the reference's f1 without materialising it: interior cells
// from the pulled values of `src`, ghost cells from `ghost` itself.
template <int Q, typename S>
__global__ void __launch_bounds__(128) k_macro(const S* __restrict__ src, const S* __restrict__ ghost, float* rho,
                                               float* u, float* v, float* w, SoaGrid g, int wrap,
                                               const S* __restrict__ xg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i > g.nx + 1) return;
    const bool interior = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
    float fp[Q];
    if (interior) {
        PullMacro<Q, S, 0>::run(fp, src, g, g.off(i, j, k), j, wrap != 0);
    } else {
        const int jw = wrap ? wrapj(j, g.ny) : j;
        const long long o = g.off(i, jw, k);
        const bool fromxg = xg && (i == 0 || i == g.nx + 1) && jw >= 1 && jw <= g.ny && k >= 1 && k <= g.nz;
#pragma unroll
        for (int l = 0; l < Q; ++l)
            fp[l] = Store<S>::to_f(fromxg ? xg[xg_index(g, Q, i == 0 ? 0 : 1, l, jw, k)] : ghost[(long long)l * g.dstride + o]);
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

namespace lbm {

// ---------------------------------------------------------------------------
// FP64 conservation sums: mass sum(rho) and momentum sum(rho u) over the
// interior cells.  Every population is converted to FP64 once and each cell's
// moments are formed and accumulated in FP64; blocks reduce with warp shuffles
// and write one partial each, a single-block kernel adds the partials in a
// fixed order.
// ---------------------------------------------------------------------------
struct Sum4 {
    double r, x, y, z;
};

// adds one cell's mass r0 + sum f_l and momentum sum c_l f_l to s, in FP64
// (each population converted once; the FP32 offsets and populations are exact in FP64)
template <int Q>
__device__ __forceinline__ void cell_sum4(Sum4& s, const float (&v)[Q], double r0) {
    double r = r0, x = 0.0, y = 0.0, z = 0.0;
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        const double d = (double)v[l];
        r += d;
        if (lat_cx(l) > 0) x += d; else if (lat_cx(l) < 0) x -= d;
        if (lat_cy(l) > 0) y += d; else if (lat_cy(l) < 0) y -= d;
        if (lat_cz(l) > 0) z += d; else if (lat_cz(l) < 0) z -= d;
    }
    s.r += r; s.x += x; s.y += y; s.z += z;
}

__device__ __forceinline__ Sum4 warp_sum4(Sum4 s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s.r += __shfl_down_sync(0xffffffffu, s.r, o);
        s.x += __shfl_down_sync(0xffffffffu, s.x, o);
        s.y += __shfl_down_sync(0xffffffffu, s.y, o);
        s.z += __shfl_down_sync(0xffffffffu, s.z, o);
    }
    return s;
}

// block reduction of per-thread sums into partial[blockIdx.x*4 .. +3]; blockDim.x = 256
__device__ __forceinline__ void block_sum4_store(Sum4 s, double* partial) {
    __shared__ double sm[8][4];
    s = warp_sum4(s);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sm[w][0] = s.r; sm[w][1] = s.x; sm[w][2] = s.y; sm[w][3] = s.z;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int q = 0; q < 8; ++q) t += sm[q][threadIdx.x];
        partial[blockIdx.x * 4 + threadIdx.x] = t;
    }
}

// interior cells of a reference-layout f(nl,0:nx+1,0:ny+1,0:nz+1)
template <int Q>
__global__ void __launch_bounds__(256) k_sum_ref(const float* __restrict__ f, RefGrid g, double* partial) {
    Sum4 s = {0.0, 0.0, 0.0, 0.0};
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long c = blockIdx.x * 256LL + threadIdx.x; c < n; c += (long long)gridDim.x * 256) {
        const int i = (int)(c % g.nx) + 1;
        const int j = (int)((c / g.nx) % g.ny) + 1;
        const int k = (int)(c / ((long long)g.nx * g.ny)) + 1;
        const float* p = f + g.cell(i, j, k) * Q;
        float v[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) v[l] = p[l];
        cell_sum4<Q>(s, v, 0.0);
    }
    block_sum4_store(s, partial);
}

// interior cells of the reference's f1 of the fused state (pulled from src)
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_sum_state(const S* __restrict__ src, SoaGrid g, int wrap, double* partial) {
    Sum4 s = {0.0, 0.0, 0.0, 0.0};
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long c = blockIdx.x * 256LL + threadIdx.x; c < n; c += (long long)gridDim.x * 256) {
        const int i = (int)(c % g.nx) + 1;
        const int j = (int)((c / g.nx) % g.ny) + 1;
        const int k = (int)(c / ((long long)g.nx * g.ny)) + 1;
        float fp[Q];
        PullMacro<Q, S, 0>::run(fp, src, g, g.off(i, j, k), j, wrap != 0);
        cell_sum4<Q>(s, fp, 1.0);     // f = f' + w_l and sum w_l = 1
    }
    block_sum4_store(s, partial);
}

// interior cells of a stored state buffer as it is (an imported f1, before any step)
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_sum_stored(const S* __restrict__ src, SoaGrid g, double* partial) {
    Sum4 s = {0.0, 0.0, 0.0, 0.0};
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long c = blockIdx.x * 256LL + threadIdx.x; c < n; c += (long long)gridDim.x * 256) {
        const int i = (int)(c % g.nx) + 1;
        const int j = (int)((c / g.nx) % g.ny) + 1;
        const int k = (int)(c / ((long long)g.nx * g.ny)) + 1;
        float fp[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) fp[l] = Store<S>::to_f(src[(long long)l * g.dstride + g.off(i, j, k)]);
        cell_sum4<Q>(s, fp, 1.0);
    }
    block_sum4_store(s, partial);
}

__global__ void __launch_bounds__(256) k_sum_final(const double* __restrict__ partial, int nblocks, double* out) {
    Sum4 s = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += 256) {
        s.r += partial[b * 4 + 0]; s.x += partial[b * 4 + 1]; s.y += partial[b * 4 + 2]; s.z += partial[b * 4 + 3];
    }
    __shared__ double sm[8][4];
    s = warp_sum4(s);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sm[w][0] = s.r; sm[w][1] = s.x; sm[w][2] = s.y; sm[w][3] = s.z;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int q = 0; q < 8; ++q) t += sm[q][threadIdx.x];
        out[threadIdx.x] = t;
    }
}

}  // namespace lbm
