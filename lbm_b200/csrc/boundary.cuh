// boundary.cuh -- ghost-cell kernels of boundarycond (m_boundarycond.F90:14-468),
// written once against a layout accessor so that the per-call entry point
// (reference layout) and the fused state (structure of arrays) share them.
//
// Every kernel here reads and writes ghost cells only from the interior or
// from the previous buffer, so threads never race: a closed-face thread writes
// its own ghost cell and reads the interior plane; periodic threads copy whole
// planes one element each.
#pragma once

#include "common.cuh"

namespace lbm {

// Accessor for the reference layout f(nl,0:nx+1,0:ny+1,0:nz+1), absolute values
// in the arithmetic type R (FP32, or FP64 for the DP build's entry points).
template <typename R>
struct AosAccT {
    using real = R;
    R* f;
    RefGrid g;
    __device__ __forceinline__ R* p(int l, int i, int j, int k) const { return f + g.cell(i, j, k) * g.nl + l; }
    __device__ __forceinline__ R ld(int l, int i, int j, int k) const { return *p(l, i, j, k); }
    __device__ __forceinline__ void st(int l, int i, int j, int k, R v) const { *p(l, i, j, k) = v; }
    // this(ld,i,j,k) = s(ls,si,sj,sk)
    __device__ __forceinline__ void cp(int ld, int i, int j, int k, const AosAccT& s, int ls, int si, int sj,
                                       int sk) const {
        *p(ld, i, j, k) = *s.p(ls, si, sj, sk);
    }
};
using AosAcc = AosAccT<float>;

// Accessor for the fused state: offsets f - w_l in storage type S.
template <typename S>
struct SoaAcc {
    using real = float;
    S* f;
    SoaGrid g;
    __device__ __forceinline__ S* p(int l, int i, int j, int k) const { return f + (long long)l * g.dstride + g.off(i, j, k); }
    __device__ __forceinline__ float ld(int l, int i, int j, int k) const { return Store<S>::to_f(*p(l, i, j, k)); }
    __device__ __forceinline__ void st(int l, int i, int j, int k, float v) const { *p(l, i, j, k) = Store<S>::from_f(v); }
    // this(ld,i,j,k) = s(ls,si,sj,sk), copied in storage type (exact)
    __device__ __forceinline__ void cp(int ld, int i, int j, int k, const SoaAcc& s, int ls, int si, int sj,
                                       int sk) const {
        *p(ld, i, j, k) = *s.p(ls, si, sj, sk);
    }
};

// Up to 9 (outgoing l, reflected m) pairs of one closed face, computed on the
// host by the reference's first-match search (m_boundary_k_closed_kernel.F90:35-46).
struct FacePairs {
    int n;
    int8_t l[9], m[9];
    int8_t cx[9], cy[9], cz[9];   // components of c_l
};

// One of the three periodic copies (m_boundary_{i,j,k}_periodic_kernel.F90).
// axis 0: i, 1: j, 2: k.  Grid: x over the fastest remaining index, y over the
// other, z over l.
template <typename Acc>
__global__ void k_periodic(Acc a, int axis, int nl) {
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int l = blockIdx.z;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (l >= nl) return;
    if (axis == 0) {            // (j,k) over (0..ny+1) x (0..nz+1); t = j, s = k
        if (t > ny + 1) return;
        a.cp(l, 0, t, s, a, l, nx, t, s);
        a.cp(l, nx + 1, t, s, a, l, 1, t, s);
    } else if (axis == 1) {     // t = i, s = k
        if (t > nx + 1) return;
        a.cp(l, t, 0, s, a, l, t, ny, s);
        a.cp(l, t, ny + 1, s, a, l, t, 1, s);
    } else {                    // t = i, s = j
        if (t > nx + 1) return;
        a.cp(l, t, s, 0, a, l, t, s, nz);
        a.cp(l, t, s, nz + 1, a, l, t, s, 1);
    }
}

// Closed faces of one axis, both sides in one launch (blockIdx.z = side).
// For each outgoing l: f1(m,ghost) = f2(l,ghost); f1(l,ghost) = f1(l, plane
// cell shifted by -c_l in the two tangential directions)
// (m_boundary_{i,j,k}_closed_kernel.F90).
template <typename Acc>
__global__ void k_closed(Acc f1, Acc f2, int axis, FacePairs lo, FacePairs hi, int lo_on, int hi_on) {
    const int nx = f1.g.nx, ny = f1.g.ny, nz = f1.g.nz;
    const int side = blockIdx.z;
    if ((side == 0 && !lo_on) || (side == 1 && !hi_on)) return;
    const FacePairs& fp = side ? hi : lo;
    const int a = blockIdx.x * blockDim.x + threadIdx.x + 1;   // first tangential index, 1-based
    const int b = blockIdx.y + 1;                              // second tangential index
    int i, j, k, pi, pj, pk;
    if (axis == 0) {           // tangential (j, k)
        if (a > ny) return;
        j = a; k = b; i = side ? nx + 1 : 0; pi = side ? nx : 1; pj = j; pk = k;
    } else if (axis == 1) {    // tangential (i, k)
        if (a > nx) return;
        i = a; k = b; j = side ? ny + 1 : 0; pj = side ? ny : 1; pi = i; pk = k;
    } else {                   // tangential (i, j)
        if (a > nx) return;
        i = a; j = b; k = side ? nz + 1 : 0; pk = side ? nz : 1; pi = i; pj = j;
    }
    for (int q = 0; q < fp.n; ++q) {
        const int l = fp.l[q], m = fp.m[q];
        f1.cp(m, i, j, k, f2, l, i, j, k);
        const int si = (axis == 0) ? pi : pi - fp.cx[q];
        const int sj = (axis == 1) ? pj : pj - fp.cy[q];
        const int sk = (axis == 2) ? pk : pk - fp.cz[q];
        f1.cp(l, i, j, k, f1, l, si, sj, sk);
    }
}

// Edges of two closed axes (m_boundary_{j_k,i_j,i_k}_edges.F90): up to four
// edges per launch (blockIdx.y), a thread per cell along the free axis.
struct EdgeDesc {
    int gi, gj, gk;        // ghost coordinates (-1 marks the free axis)
    int si, sj, sk;        // source coordinates of pass 2 (-1 marks the free axis)
    int n;                 // number of outgoing directions
    int8_t l[3], m[3];
};
struct EdgeSet {
    int free_axis, nfree, nedges;
    EdgeDesc e[4];
};

template <typename Acc>
__global__ void k_edges(Acc f1, Acc f2, EdgeSet es) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (t > es.nfree || blockIdx.y >= es.nedges) return;
    const EdgeDesc& d = es.e[blockIdx.y];
    const int i = d.gi < 0 ? t : d.gi, j = d.gj < 0 ? t : d.gj, k = d.gk < 0 ? t : d.gk;
    const int si = d.si < 0 ? t : d.si, sj = d.sj < 0 ? t : d.sj, sk = d.sk < 0 ? t : d.sk;
    for (int q = 0; q < d.n; ++q) f1.cp(d.m[q], i, j, k, f2, d.l[q], i, j, k);
    for (int q = 0; q < d.n; ++q) f1.cp(d.l[q], i, j, k, f1, d.l[q], si, sj, sk);
}

// The eight corners when all three axes are closed (m_boundary_closed_corners.F90).
struct CornerSet {
    int ci[8], cj[8], ck[8];
    int l[8], m[8];          // D3Q27 has one outgoing direction per corner, D3Q19 none (l = -1)
    int8_t cx[8], cy[8], cz[8];
};
template <typename Acc>
__global__ void k_corners(Acc f1, Acc f2, CornerSet cs) {
    const int t = threadIdx.x;
    if (t >= 8 || cs.l[t] < 0) return;
    const int i = cs.ci[t], j = cs.cj[t], k = cs.ck[t];
    f1.cp(cs.m[t], i, j, k, f2, cs.l[t], i, j, k);
    f1.cp(cs.l[t], i, j, k, f1, cs.l[t], i - cs.cx[t], j - cs.cy[t], k - cs.cz[t]);
}

// Inflow at i=0 and zero-gradient outflow at i=nx+1, m_boundary_i_inflow_kernel.F90:56-111.
// fghost(l) = f(l,1,j,k) - 2 w_l rho0 (cx u cos + cy u sin) / cs2; directions with
// cx > 0 take fghost of their opposite.  In offset storage w_l cancels, and
// opposite directions share w_l, so the same update holds for f - w_l.
// Acc::real is the arithmetic type (FP32 for the fused state and the default
// entry point, FP64 for the DP one).
template <int Q, typename Acc>
__global__ void k_inflow(Acc f, const typename Acc::real* __restrict__ uvel, typename Acc::real rho0,
                         typename Acc::real cosd, typename Acc::real sind) {
    using R = typename Acc::real;
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int k = blockIdx.y + 1;
    const int nx = f.g.nx;
    if (j > f.g.ny) return;
    const R uu = uvel[k - 1];
    const R cs2 = R(1) / R(3);
    R fg[Q];
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        const R wl = lat_w<Q, R>(l);
        const R cxl = (R)lat_cx(l), cyl = (R)lat_cy(l);
        fg[l] = f.ld(l, 1, j, k) - R(2) * wl * rho0 * (cxl * uu * cosd + cyl * uu * sind) / cs2;
    }
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        const R v = (lat_cx(l) <= 0) ? fg[l] : fg[lat_opposite(l)];
        f.st(l, 0, j, k, v);
    }
#pragma unroll
    for (int l = 0; l < Q; ++l) f.cp(l, nx + 1, j, k, f, l, nx, j, k);
}

}  // namespace lbm
