// common.cuh -- lattice tables, grid layouts and storage traits shared by the
// kernels of the B200 LBM library.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace lbm {

// ---------------------------------------------------------------------------
// Lattice tables in the reference's direction order (mod_D3Q27setup.F90:28-48).
// D3Q19 is the first 19 directions of D3Q27.  Directions 2k-1 and 2k
// (0-based, k >= 1) are opposite, which both the solid swap (m_solids.F90:28-32)
// and the pairwise evaluation of the collision rely on.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int lat_cx(int l) {
    constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1};
    return t[l];
}
__host__ __device__ constexpr int lat_cy(int l) {
    constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 0, 0, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
    return t[l];
}
__host__ __device__ constexpr int lat_cz(int l) {
    constexpr int t[27] = {0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1};
    return t[l];
}
__host__ __device__ constexpr int lat_speed2(int l) {
    return lat_cx(l) * lat_cx(l) + lat_cy(l) * lat_cy(l) + lat_cz(l) * lat_cz(l);
}
// weights: D3Q19 {1/3, 1/18, 1/36}; D3Q27 {8/27, 2/27, 1/54, 1/216}, each quotient
// rounded once in the arithmetic type R (FP32, or FP64 as the reference's DP build)
template <int Q, typename R = float>
__host__ __device__ constexpr R lat_w(int l) {
    return Q == 19 ? (lat_speed2(l) == 0 ? R(1) / R(3) : lat_speed2(l) == 1 ? R(1) / R(18) : R(1) / R(36))
                   : (lat_speed2(l) == 0 ? R(8) / R(27)
                      : lat_speed2(l) == 1 ? R(2) / R(27)
                      : lat_speed2(l) == 2 ? R(1) / R(54)
                                           : R(1) / R(216));
}
// tiny(1.0) of the arithmetic type: the smallest positive normal number
template <typename R>
__host__ __device__ constexpr R lat_tiny();
template <>
__host__ __device__ constexpr float lat_tiny<float>() { return 1.17549435e-38f; }
template <>
__host__ __device__ constexpr double lat_tiny<double>() { return 2.2250738585072014e-308; }
// square root and maximum in the arithmetic type (sqrtf / fmaxf for FP32)
__device__ __forceinline__ float real_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double real_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float real_max(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double real_max(double a, double b) { return fmax(a, b); }
__host__ __device__ constexpr int lat_opposite(int l) { return l == 0 ? 0 : ((l & 1) ? l + 1 : l - 1); }
// index of direction (x,y,z) among the first Q directions, -1 if absent
template <int Q>
__host__ __device__ constexpr int lat_find(int x, int y, int z) {
    for (int m = 0; m < Q; ++m)
        if (lat_cx(m) == x && lat_cy(m) == y && lat_cz(m) == z) return m;
    return -1;
}

// The same tables in constant memory, for kernels that index directions at run time.
#define LBM_27(F) F(0), F(1), F(2), F(3), F(4), F(5), F(6), F(7), F(8), F(9), F(10), F(11), F(12), F(13), \
    F(14), F(15), F(16), F(17), F(18), F(19), F(20), F(21), F(22), F(23), F(24), F(25), F(26)
#define LBM_CX(l) lat_cx(l)
#define LBM_CY(l) lat_cy(l)
#define LBM_CZ(l) lat_cz(l)
#define LBM_OPP(l) lat_opposite(l)
#define LBM_W19(l) lat_w<19>(l)
#define LBM_W27(l) lat_w<27>(l)
__constant__ int8_t c_cx[27] = {LBM_27(LBM_CX)};
__constant__ int8_t c_cy[27] = {LBM_27(LBM_CY)};
__constant__ int8_t c_cz[27] = {LBM_27(LBM_CZ)};
__constant__ int8_t c_opp[27] = {LBM_27(LBM_OPP)};
__constant__ float c_w[2][27] = {{LBM_27(LBM_W19)}, {LBM_27(LBM_W27)}};   // [0] D3Q19, [1] D3Q27

// Programmatic dependent launch (PDL) between consecutive kernels of a stream
// (the steady step kernel and the boundary kernel, the kernels of a reverse
// step): each kernel lets the next one in the stream be scheduled as soon as
// all its own blocks have started, and every thread of the next one
// waits at its start until the previous grid has completed and its memory is
// visible.  Launched without the PDL attribute, both instructions do nothing.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Reference layout f(nl,0:nx+1,0:ny+1,0:nz+1), l fastest (Fortran column-major).
// ---------------------------------------------------------------------------
struct RefGrid {
    int nx, ny, nz, nl;
    __host__ __device__ long long cell(int i, int j, int k) const {
        return (long long)i + (long long)(nx + 2) * ((long long)j + (long long)(ny + 2) * k);
    }
    __host__ __device__ long long ncell() const { return (long long)(nx + 2) * (ny + 2) * (nz + 2); }
};

// ---------------------------------------------------------------------------
// Structure-of-arrays layout of the fused state.  Each direction is a block of
// (ny+2)*(nz+2) rows of `pitch` elements; in a row, ghost i=0 sits at offset
// 31 so that the interior i=1..nx starts on a 128-byte boundary (FP32) and a
// warp of consecutive i writes whole cache lines.  pitch = roundup(nx+34, 32)
// leaves at least 34 elements of padding per row, so that (for nx a multiple
// of the sector's element count) the 32-byte sectors holding ghost i=0 and
// ghost nx+1 contain nothing else: the boundary kernel writes them whole.
// ---------------------------------------------------------------------------
struct SoaGrid {
    int nx, ny, nz;
    int pitch;            // elements per row
    long long rowsz;      // elements per (j,k) row block = pitch
    long long dstride;    // elements per direction
    __host__ __device__ int row(int j, int k) const { return k * (ny + 2) + j; }
    // element offset of cell (i,j,k) inside a direction block (i,j,k ghost-inclusive)
    __host__ __device__ long long off(int i, int j, int k) const {
        return (long long)row(j, k) * pitch + 31 + i;
    }
    static SoaGrid make(int nx, int ny, int nz) {
        SoaGrid g;
        g.nx = nx; g.ny = ny; g.nz = nz;
        g.pitch = ((nx + 34 + 31) / 32) * 32;
        g.rowsz = g.pitch;
        g.dstride = (long long)(ny + 2) * (nz + 2) * g.pitch + 32;
        return g;
    }
};

// ---------------------------------------------------------------------------
// Storage traits: the fused state stores f' = f - w_l, the offset from the
// rest-state weight, either in FP32 or as FP16 scaled by 2^8.  The offset
// form keeps the small non-equilibrium part away from the large constant w_l,
// which costs nothing in FP32 and is what makes FP16 storage usable.
// ---------------------------------------------------------------------------
template <typename S>
struct Store;
template <>
struct Store<float> {
    static __device__ __forceinline__ float load(const float* p) { return __ldg(p); }
    static __device__ __forceinline__ void store(float* p, float v) { *p = v; }
    static __host__ __device__ __forceinline__ float to_f(float s) { return s; }
    static __host__ __device__ __forceinline__ float from_f(float v) { return v; }
};
template <>
struct Store<__half> {
    static __device__ __forceinline__ float load(const __half* p) { return __half2float(__ldg(p)) * (1.0f / 256.0f); }
    static __device__ __forceinline__ void store(__half* p, float v) { *p = __float2half_rn(v * 256.0f); }
    static __device__ __forceinline__ float to_f(__half s) { return __half2float(s) * (1.0f / 256.0f); }
    static __device__ __forceinline__ __half from_f(float v) { return __float2half_rn(v * 256.0f); }
};

}  // namespace lbm
