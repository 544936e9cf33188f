// turbulence.cuh -- inflow-turbulence fields on the GPU
// (m_inflow_turbulence_compute.F90:3-62 with m_pseudo2D.F90:3-169).
//
// Each level of each field is a 2-D Gaussian random field on the (j, k) plane:
// Fourier amplitudes e(l,p) = exp(-(a11 kappa^2 l^2 + a22 lambda^2 p^2)) with
// uniformly random phases, scaled so the field variance is one
// (m_pseudo2D.F90:96-143), synthesised by a complex-to-real FFT (cuFFT here,
// FFTW there).  The levels 1..nrturb are then chained by the AR(1) relation
// x_t = 0.98 x_(t-1) + sqrt(1 - 0.98^2) x_t and each is normalised to zero mean
// and unit sample standard deviation (m_inflow_turbulence_compute.F90:35-60).
//
// The phases come from SplitMix64 (Steele, Lea and Flood 2014; the finaliser
// of Vigna's splitmix64) applied to a counter built from the seed, the field,
// the level and the wavenumber, instead of the compiler's random_number.  The
// wavenumber columns l = 0 and l = n1/2 are made Hermitian (x(l,-p) =
// conj(x(l,p)), real at the self-conjugate points), so the real transform is
// well defined whatever FFT library runs it.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace lbm {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// uniform in [0, 1) with 24 random bits
__host__ __device__ __forceinline__ float unit_uniform(uint64_t seed, uint64_t counter) {
    return (float)(splitmix64(seed ^ splitmix64(counter)) >> 40) * (1.0f / 16777216.0f);
}

struct TurbSpec {
    int n1, n2;          // FFT grid (ny, nz rounded up to even)
    int nb;              // fields x levels
    float amp;           // sqrt(deltak) * c
    float ak, al;        // a11 kappa^2, a22 lambda^2
    uint64_t seed;
};

// X[b][p_idx][l], l = 0..n1/2, p_idx = 0..n2-1 (p = p_idx, or p_idx - n2 above n2/2 - 1)
__global__ void k_turb_spectrum(float2* X, TurbSpec s) {
    const int h = s.n1 / 2 + 1;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)s.nb * s.n2 * h;
    if (e >= n) return;
    const int l = (int)(e % h);
    const int pi = (int)((e / h) % s.n2);
    const int b = (int)(e / ((long long)h * s.n2));
    int p = pi < s.n2 / 2 ? pi : pi - s.n2;
    // Hermitian columns: the value at -p is the conjugate of the one at p
    const bool herm = (l == 0 || l == s.n1 / 2);
    float sgn = 1.0f;
    bool real_only = false;
    if (herm) {
        if (p < 0 && p != -s.n2 / 2) {
            p = -p;
            sgn = -1.0f;
        }
        real_only = (p == 0 || p == -s.n2 / 2);
    }
    const uint64_t counter = ((uint64_t)b * (uint64_t)(s.n2 + 1) + (uint64_t)(p + s.n2 / 2)) * (uint64_t)h + (uint64_t)l;
    const float phi = 6.283185307179586f * unit_uniform(s.seed, counter);
    const float ee = s.amp * expf(-(s.ak * (float)(l * l) + s.al * (float)(p * p)));
    float re = ee * cosf(phi), im = sgn * ee * sinf(phi);
    if (real_only) im = 0.0f;
    if (l == 0 && p == 0) re = 0.0f;   // lmean = .false.: no mean in any realisation
    X[e] = make_float2(re, im);
}

// One block per field: copy the level fields out of the FFT grid, then chain
// and normalise levels 1..nrturb in order.  out[t][k-1][j-1] (ny, nz, 0:nrturb).
template <int NT>
__global__ void __launch_bounds__(NT) k_turb_ar1(const float* Y, float* const* outs, int ny, int nz, int n1, int n2,
                                                  int nrturb) {
    __shared__ double red[NT / 32][2];
    float* out = outs[blockIdx.x];
    const long long plane = (long long)ny * nz;
    const float tc = 0.98f, tn = sqrtf(1.0f - 0.98f * 0.98f);
    for (int t = 0; t <= nrturb; ++t) {
        const float* y = Y + ((long long)blockIdx.x * (nrturb + 1) + t) * n1 * n2;
        float* o = out + (long long)t * plane;
        double s = 0.0;
        for (long long e = threadIdx.x; e < plane; e += NT) {
            const int j = (int)(e % ny), k = (int)(e / ny);
            float v = y[(long long)k * n1 + j];      // Amat(j, k) = y(j-1, k-1), first FFT index fastest
            if (t > 0) v = tc * o[e - plane] + tn * v;
            o[e] = v;
            s += v;
        }
        if (t == 0) continue;
        // mean, then sample standard deviation, over the plane (accumulated in FP64)
        for (int pass = 0; pass < 2; ++pass) {
            for (int q = 16; q > 0; q >>= 1) s += __shfl_down_sync(0xffffffffu, s, q);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][pass] = s;
            __syncthreads();
            double tot = 0.0;
            for (int w = 0; w < NT / 32; ++w) tot += red[w][pass];
            __syncthreads();
            if (pass == 0) {
                const float mean = (float)(tot / (double)plane);
                s = 0.0;
                for (long long e = threadIdx.x; e < plane; e += NT) {
                    const float v = o[e] - mean;
                    o[e] = v;
                    s += (double)v * (double)v;
                }
            } else {
                const float inv = (float)(1.0 / sqrt(tot / (double)(plane - 1)));
                for (long long e = threadIdx.x; e < plane; e += NT) o[e] *= inv;
            }
        }
    }
}

}  // namespace lbm
