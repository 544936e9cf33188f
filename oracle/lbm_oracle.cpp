// lbm_oracle.cpp -- CPU oracle for the LBM per-timestep path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, routine by routine, the
// arithmetic of geirev/LBM (src/*.F90) so that the CUDA library can be checked
// against it.  Only tests/, __graft_entry__.smoke() and the CPU legs of
// bench.py (the CPU baseline and the reference arm) load it; the product
// library never does.
//
// Parity status: UNPINNED against reference outputs (the reference ships no
// golden vectors and needs a Fortran compiler this image lacks).  It is pinned
// by analytic known answers and by an independent numpy restatement
// (tests/golden/make_golden.py); see tests/test_oracle_*.py.
//
// Every loop keeps the reference's loop nesting and summation order so that the
// FP32 instantiation (built with -ffp-contract=off) rounds like the reference's
// single-precision CPU build, and the FP64 instantiation follows its DP=1
// (-r8) build, where every default-real constant, tiny() and eps included, is
// double precision.
#include "lbm_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// Lattice tables, mod_D3Q27setup.F90:28-48 (D3Q19 :28-35, D3Q27 :40-48).
// Stored 0-based here; the reference arrays are 1-based.
// ---------------------------------------------------------------------------
const int CX19[19] = {0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1,-1, 1, 0, 0,-1, 1, 0, 0};
const int CY19[19] = {0, 0, 0, 1,-1, 0, 0, 1,-1,-1, 1, 0, 0, 1,-1, 0, 0,-1, 1};
const int CZ19[19] = {0, 0, 0, 0, 0,-1, 1, 0, 0, 0, 0,-1, 1, 1,-1, 1,-1, 1,-1};
const int CX27[27] = {0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1,-1, 1, 0, 0,-1, 1, 0, 0,-1, 1,-1, 1, 1,-1,-1, 1};
const int CY27[27] = {0, 0, 0, 1,-1, 0, 0, 1,-1,-1, 1, 0, 0, 1,-1, 0, 0,-1, 1, 1,-1,-1, 1, 1,-1, 1,-1};
const int CZ27[27] = {0, 0, 0, 0, 0,-1, 1, 0, 0, 0, 0,-1, 1, 1,-1, 1,-1, 1,-1, 1,-1,-1, 1,-1, 1,-1, 1};

template <typename T>
struct Lattice {
    int nl;
    int cx[27], cy[27], cz[27], bounce[27];
    T w[27];
    T H2[27][3][3];      // H2[l][q][p] == H2(p,q,l)
    T H3[27][3][3][3];   // H3[l][r][q][p] == H3(p,q,r,l)
    T cs2, cs4, cs6, inv1cs2, inv2cs4, inv6cs6;
    T eps, tinyv;

    explicit Lattice(int q) : nl(q) {
        // mod_D3Q27setup.F90:14-16: cs2=1.0/3.0, cs4=1.0/9.0, cs6=1.0/27.0
        cs2 = T(1.0) / T(3.0);
        cs4 = T(1.0) / T(9.0);
        cs6 = T(1.0) / T(27.0);
        // m_postcoll.F90:40-43
        inv1cs2 = T(1.0) / (cs2);
        inv2cs4 = T(1.0) / (T(2.0) * cs4);
        inv6cs6 = T(1.0) / (T(6.0) * cs6);
        tinyv = std::numeric_limits<T>::min();   // tiny(1.0)
        eps = std::sqrt(tinyv);                  // m_postcoll.F90:47
        const int* X = (q == 19) ? CX19 : CX27;
        const int* Y = (q == 19) ? CY19 : CY27;
        const int* Z = (q == 19) ? CZ19 : CZ27;
        for (int l = 0; l < q; ++l) {
            cx[l] = X[l]; cy[l] = Y[l]; cz[l] = Z[l];
            // bounce_h pairs (2,3),(4,5),... in 1-based numbering
            bounce[l] = (l == 0) ? 0 : ((l % 2 == 1) ? l + 1 : l - 1);
            int s = std::abs(X[l]) + std::abs(Y[l]) + std::abs(Z[l]);
            if (q == 19) {
                w[l] = (s == 0) ? T(1.0) / T(3.0) : (s == 1) ? T(1.0) / T(18.0) : T(1.0) / T(36.0);
            } else {
                w[l] = (s == 0) ? T(8.0) / T(27.0) : (s == 1) ? T(2.0) / T(27.0)
                     : (s == 2) ? T(1.0) / T(54.0) : T(1.0) / T(216.0);
            }
        }
        // hermite_polynomials(), mod_D3Q27setup.F90:127-150
        T c[3][27];
        for (int l = 0; l < q; ++l) { c[0][l] = T(cx[l]); c[1][l] = T(cy[l]); c[2][l] = T(cz[l]); }
        auto delta = [](int a, int b) { return a == b ? T(1.0) : T(0.0); };
        for (int l = 0; l < q; ++l)
            for (int p = 0; p < 3; ++p)
                for (int qq = 0; qq < 3; ++qq)
                    H2[l][qq][p] = c[p][l] * c[qq][l] - cs2 * delta(p, qq);
        for (int l = 0; l < q; ++l)
            for (int p = 0; p < 3; ++p)
                for (int qq = 0; qq < 3; ++qq)
                    for (int r = 0; r < 3; ++r)
                        H3[l][r][qq][p] = c[p][l] * c[qq][l] * c[r][l]
                                        - cs2 * (c[p][l] * delta(qq, r) + c[qq][l] * delta(p, r) + c[r][l] * delta(p, qq));
    }
};

struct Dims {
    int nx, ny, nz, nl;
    long nxg, nyg, nzg;
    explicit Dims(const orc_params* p)
        : nx(p->nx), ny(p->ny), nz(p->nz), nl(p->nl), nxg(p->nx + 2), nyg(p->ny + 2), nzg(p->nz + 2) {}
    // scalar field (0:nx+1,0:ny+1,0:nz+1)
    long s(long i, long j, long k) const { return i + nxg * (j + nyg * k); }
    // distribution f(nl,0:nx+1,0:ny+1,0:nz+1), l 0-based
    long f(long l, long i, long j, long k) const { return l + nl * s(i, j, k); }
    long ncell() const { return nxg * nyg * nzg; }
};

// ---------------------------------------------------------------------------
// fequil3_kernel, m_fequil3_kernel.F90:58-123 (interior only)
// ---------------------------------------------------------------------------
template <typename T>
void fequil3(const orc_params* p, T* feq, const T* rho, const T* u, const T* v, const T* w) {
    const Lattice<T> L(p->nl);
    const Dims d(p);
    const T ratio = L.inv6cs6 / L.inv2cs4;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j)
            for (int i = 1; i <= d.nx; ++i) {
                long c = d.s(i, j, k);
                T vel[3] = {u[c], v[c], w[c]};
                T dens = rho[c];
                T A2[3][3], A3[3][3][3];
                for (int q = 0; q < 3; ++q)
                    for (int pp = 0; pp < 3; ++pp) A2[q][pp] = dens * vel[pp] * vel[q] * L.inv2cs4;
                if (p->ibgk == 3)
                    for (int r = 0; r < 3; ++r) {
                        T vratio = vel[r] * ratio;
                        for (int q = 0; q < 3; ++q)
                            for (int pp = 0; pp < 3; ++pp) A3[r][q][pp] = A2[q][pp] * vratio;
                    }
                for (int l = 0; l < d.nl; ++l) {
                    T cu = T(L.cx[l]) * vel[0] + T(L.cy[l]) * vel[1] + T(L.cz[l]) * vel[2];
                    T tmp = dens * (T(1.0) + cu * L.inv1cs2);
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) tmp = tmp + L.H2[l][q][pp] * A2[q][pp];
                    if (p->ibgk == 3 && l > 0)
                        for (int r = 0; r < 3; ++r)
                            for (int q = 0; q < 3; ++q)
                                for (int pp = 0; pp < 3; ++pp) tmp = tmp + L.H3[l][r][q][pp] * A3[r][q][pp];
                    feq[d.f(l, i, j, k)] = L.w[l] * tmp;
                }
            }
}

// ---------------------------------------------------------------------------
// postcoll_kernel, m_postcoll_kernel.F90:7-255 (equilibrium :70-117,
// regularization :123-185, Vreman :189-239, BGK update :242-245)
// ---------------------------------------------------------------------------
template <typename T>
void postcoll(const orc_params* p, T* f, T* tau, const T* rho, const T* u, const T* v, const T* w, const T* ablvisc) {
    const Lattice<T> L(p->nl);
    const Dims d(p);
    const T ratio = L.inv6cs6 / L.inv2cs4;
    const T kinevisc = T(p->kinevisc);
    const T smag = T(p->smagorinsky);
    const T cnst = T(2.5) * smag * smag;   // m_postcoll.F90:46 const=2.5*smagorinsky**2
    const T eps = L.eps;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j)
            for (int i = 1; i <= d.nx; ++i) {
                long c = d.s(i, j, k);
                T vel[3] = {u[c], v[c], w[c]};
                T dens = rho[c];
                T A2[3][3], A3[3][3][3];
                T tmpeq[27], tmpneq[27];
                for (int q = 0; q < 3; ++q)
                    for (int pp = 0; pp < 3; ++pp) A2[q][pp] = dens * vel[pp] * vel[q] * L.inv2cs4;
                if (p->ibgk == 3)
                    for (int r = 0; r < 3; ++r) {
                        T vratio = vel[r] * ratio;
                        for (int q = 0; q < 3; ++q)
                            for (int pp = 0; pp < 3; ++pp) A3[r][q][pp] = A2[q][pp] * vratio;
                    }
                for (int l = 0; l < d.nl; ++l) {
                    T cu = T(L.cx[l]) * vel[0] + T(L.cy[l]) * vel[1] + T(L.cz[l]) * vel[2];
                    tmpeq[l] = dens * (T(1.0) + cu * L.inv1cs2);
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) tmpeq[l] = tmpeq[l] + L.H2[l][q][pp] * A2[q][pp];
                    if (p->ibgk == 3 && l > 0)
                        for (int r = 0; r < 3; ++r)
                            for (int q = 0; q < 3; ++q)
                                for (int pp = 0; pp < 3; ++pp) tmpeq[l] = tmpeq[l] + L.H3[l][r][q][pp] * A3[r][q][pp];
                    tmpeq[l] = L.w[l] * tmpeq[l];
                }
                if (p->ihrr == 1) {
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) A2[q][pp] = T(0.0);
                    for (int l = 0; l < d.nl; ++l) {
                        tmpneq[l] = f[d.f(l, i, j, k)] - tmpeq[l];
                        for (int q = 0; q < 3; ++q)
                            for (int pp = 0; pp < 3; ++pp) A2[q][pp] = A2[q][pp] + L.H2[l][q][pp] * tmpneq[l];
                    }
                    // A3(p,q,r)=vel(p)*A2(q,r) + vel(q)*A2(r,p) + vel(r)*A2(p,q)   (:202-208)
                    for (int r = 0; r < 3; ++r)
                        for (int q = 0; q < 3; ++q)
                            for (int pp = 0; pp < 3; ++pp)
                                A3[r][q][pp] = vel[pp] * A2[r][q] + vel[q] * A2[pp][r] + vel[r] * A2[q][pp];
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) A2[q][pp] = A2[q][pp] * L.inv2cs4;
                    for (int r = 0; r < 3; ++r)
                        for (int q = 0; q < 3; ++q)
                            for (int pp = 0; pp < 3; ++pp) A3[r][q][pp] = A3[r][q][pp] * L.inv6cs6;
                    for (int l = 0; l < d.nl; ++l) {
                        T t = T(0.0);
                        for (int q = 0; q < 3; ++q)
                            for (int pp = 0; pp < 3; ++pp) t = t + L.H2[l][q][pp] * A2[q][pp];
                        for (int r = 0; r < 3; ++r)
                            for (int q = 0; q < 3; ++q)
                                for (int pp = 0; pp < 3; ++pp) t = t + L.H3[l][r][q][pp] * A3[r][q][pp];
                        tmpneq[l] = L.w[l] * t;
                    }
                } else {
                    for (int l = 0; l < d.nl; ++l) tmpneq[l] = f[d.f(l, i, j, k)] - tmpeq[l];
                }
                if (p->ivreman == 1) {
                    T alpha[3][3];   // alpha[q][p] == alpha(p,q)
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) alpha[q][pp] = T(0.0);
                    for (int l = 0; l < d.nl; ++l)
                        for (int q = 0; q < 3; ++q)
                            for (int pp = 0; pp < 3; ++pp) alpha[q][pp] = alpha[q][pp] + L.H2[l][q][pp] * tmpneq[l];
                    T alphamag = T(0.0);
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) alphamag = alphamag + alpha[q][pp] * alpha[q][pp];
                    alphamag = std::max(alphamag, L.tinyv);
                    T beta[3][3];    // beta[q][p] == beta(p,q)
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) {
                            beta[q][pp] = eps;
                            for (int m = 0; m < 3; ++m) beta[q][pp] = beta[q][pp] + alpha[pp][m] * alpha[q][m];
                        }
                    // Bbeta=b11*b22-b12**2+b11*b33-b13**2+b22*b33-b23**2 (left to right)
                    T b11 = beta[0][0], b22 = beta[1][1], b33 = beta[2][2];
                    T b12 = beta[1][0], b13 = beta[2][0], b23 = beta[2][1];
                    T Bbeta = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
                    T tautmp = Bbeta / alphamag;
                    T eddyvisc = (tautmp > eps) ? cnst * std::sqrt(tautmp) : T(0.0);
                    tau[c] = T(3.0) * (kinevisc + eddyvisc + ablvisc[k - 1]) + T(0.5);
                }
                T fac = T(1.0) - T(1.0) / tau[c];
                for (int l = 0; l < d.nl; ++l) f[d.f(l, i, j, k)] = tmpeq[l] + fac * tmpneq[l];
            }
}

// ---------------------------------------------------------------------------
// drift_kernel, m_drift_kernel.F90:37-42: f(l,i,j,k) = feq(l,i-cx,j-cy,k-cz)
// ---------------------------------------------------------------------------
template <typename T>
void drift(const orc_params* p, T* f, const T* feq) {
    const Lattice<T> L(p->nl);
    const Dims d(p);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j)
            for (int i = 1; i <= d.nx; ++i)
                for (int l = 0; l < d.nl; ++l)
                    f[d.f(l, i, j, k)] = feq[d.f(l, i - L.cx[l], j - L.cy[l], k - L.cz[l])];
}

// ---------------------------------------------------------------------------
// macrovars_kernel, m_macrovars_kernel.F90:35-49 (over the ghost shell too)
// ---------------------------------------------------------------------------
template <typename T>
void macrovars(const orc_params* p, T* rho, T* u, T* v, T* w, const T* f) {
    const Lattice<T> L(p->nl);
    const Dims d(p);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k <= d.nz + 1; ++k)
        for (int j = 0; j <= d.ny + 1; ++j)
            for (int i = 0; i <= d.nx + 1; ++i) {
                T tr = T(0.0), tu = T(0.0), tv = T(0.0), tw = T(0.0);
                for (int l = 0; l < d.nl; ++l) {
                    T tf = f[d.f(l, i, j, k)];
                    tr = tr + tf;
                    tu = tu + T(L.cx[l]) * tf;
                    tv = tv + T(L.cy[l]) * tf;
                    tw = tw + T(L.cz[l]) * tf;
                }
                T invrho = T(1.0) / tr;
                long c = d.s(i, j, k);
                rho[c] = tr;
                u[c] = tu * invrho;
                v[c] = tv * invrho;
                w[c] = tw * invrho;
            }
}

// ---------------------------------------------------------------------------
// regularization_kernel, m_regularization_kernel.F90:44-113 (output: R(fneq))
// ---------------------------------------------------------------------------
template <typename T>
void regularization(const orc_params* p, T* f, const T* feq, const T* u, const T* v, const T* w) {
    const Lattice<T> L(p->nl);
    const Dims d(p);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j)
            for (int i = 1; i <= d.nx; ++i) {
                long c = d.s(i, j, k);
                T vel[3] = {u[c], v[c], w[c]};
                T a2[3][3], a3[3][3][3];
                for (int q = 0; q < 3; ++q)
                    for (int pp = 0; pp < 3; ++pp) a2[q][pp] = T(0.0);
                for (int l = 0; l < d.nl; ++l) {
                    T tmp = f[d.f(l, i, j, k)] - feq[d.f(l, i, j, k)];
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) a2[q][pp] = a2[q][pp] + L.H2[l][q][pp] * tmp;
                }
                for (int r = 0; r < 3; ++r)
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp)
                            a3[r][q][pp] = vel[pp] * a2[r][q] + vel[q] * a2[pp][r] + vel[r] * a2[q][pp];
                for (int q = 0; q < 3; ++q)
                    for (int pp = 0; pp < 3; ++pp) a2[q][pp] = a2[q][pp] * L.inv2cs4;
                for (int r = 0; r < 3; ++r)
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) a3[r][q][pp] = a3[r][q][pp] * L.inv6cs6;
                for (int l = 0; l < d.nl; ++l) {
                    T tmp = T(0.0);
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) tmp = tmp + L.H2[l][q][pp] * a2[q][pp];
                    for (int r = 0; r < 3; ++r)
                        for (int q = 0; q < 3; ++q)
                            for (int pp = 0; pp < 3; ++pp) tmp = tmp + L.H3[l][r][q][pp] * a3[r][q][pp];
                    f[d.f(l, i, j, k)] = L.w[l] * tmp;
                }
            }
}

// ---------------------------------------------------------------------------
// vreman_kernel, m_vreman_kernel.F90:47-91 (standalone guards: 1e-5 offsets,
// no ablvisc, no max(.,tiny))
// ---------------------------------------------------------------------------
template <typename T>
void vreman(const orc_params* p, const T* f, T* tau) {
    if (p->ivreman != 1) return;   // m_vreman.F90:29-31
    const Lattice<T> L(p->nl);
    const Dims d(p);
    const T kinevisc = T(p->kinevisc);
    const T smag = T(p->smagorinsky);
    const T cnst = T(2.5) * smag * smag;
    const T eps = L.eps;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j)
            for (int i = 1; i <= d.nx; ++i) {
                T alpha[3][3];
                for (int q = 0; q < 3; ++q)
                    for (int pp = 0; pp < 3; ++pp) alpha[q][pp] = T(0.0);
                for (int l = 0; l < d.nl; ++l) {
                    T tmp = f[d.f(l, i, j, k)];
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) alpha[q][pp] = alpha[q][pp] + L.H2[l][q][pp] * tmp;
                }
                T alphamag = T(0.00001);
                for (int q = 0; q < 3; ++q)
                    for (int pp = 0; pp < 3; ++pp) alphamag = alphamag + alpha[q][pp] * alpha[q][pp];
                T beta[3][3];
                for (int q = 0; q < 3; ++q)
                    for (int pp = 0; pp < 3; ++pp) {
                        beta[q][pp] = T(0.00001);
                        for (int m = 0; m < 3; ++m) beta[q][pp] = beta[q][pp] + alpha[pp][m] * alpha[q][m];
                    }
                T b11 = beta[0][0], b22 = beta[1][1], b33 = beta[2][2];
                T b12 = beta[1][0], b13 = beta[2][0], b23 = beta[2][1];
                T Bbeta = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
                T tmp = Bbeta / alphamag;
                T eddyvisc = (tmp > eps) ? cnst * std::sqrt(tmp) : T(0.0);
                tau[d.s(i, j, k)] = T(3.0) * (kinevisc + eddyvisc) + T(0.5);
            }
}

// compute_fneq_kernel / compute_f_kernel: flat over every element incl. ghosts
template <typename T>
void compute_fneq(const orc_params* p, T* f, const T* feq) {
    const Dims d(p);
    long n = d.ncell() * d.nl;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) f[i] = f[i] - feq[i];
}
template <typename T>
void compute_f(const orc_params* p, T* f, const T* feq) {
    const Dims d(p);
    long n = d.ncell() * d.nl;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) f[i] = feq[i] + f[i];
}

// ---------------------------------------------------------------------------
// Boundary kernels, m_boundary_*_kernel.F90 and the CUF edge/corner loops
// ---------------------------------------------------------------------------
template <typename T>
int find_dir(const Lattice<T>& L, int mx, int my, int mz) {
    for (int m = 0; m < L.nl; ++m)
        if (L.cx[m] == mx && L.cy[m] == my && L.cz[m] == mz) return m;
    return -1;
}

// m_boundary_i_periodic_kernel.F90:30-33
template <typename T>
void bnd_i_periodic(const Dims& d, T* f) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k <= d.nz + 1; ++k)
        for (int j = 0; j <= d.ny + 1; ++j)
            for (int l = 0; l < d.nl; ++l) {
                f[d.f(l, 0, j, k)] = f[d.f(l, d.nx, j, k)];
                f[d.f(l, d.nx + 1, j, k)] = f[d.f(l, 1, j, k)];
            }
}
// m_boundary_j_periodic_kernel.F90:30-33
template <typename T>
void bnd_j_periodic(const Dims& d, T* f) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k <= d.nz + 1; ++k)
        for (int i = 0; i <= d.nx + 1; ++i)
            for (int l = 0; l < d.nl; ++l) {
                f[d.f(l, i, 0, k)] = f[d.f(l, i, d.ny, k)];
                f[d.f(l, i, d.ny + 1, k)] = f[d.f(l, i, 1, k)];
            }
}
// m_boundary_k_periodic_kernel.F90:13-27
template <typename T>
void bnd_k_periodic(const Dims& d, T* f) {
    long plane = d.nl * d.nxg * d.nyg;
    T* p0 = f;
    T* p1 = f + plane;
    T* pn = f + plane * d.nz;
    T* pn1 = f + plane * (d.nz + 1);
    for (long i = 0; i < plane; ++i) {
        p0[i] = pn[i];
        pn1[i] = p1[i];
    }
}
// m_boundary_i_closed_kernel.F90:31-58
template <typename T>
void bnd_i_closed(const Lattice<T>& L, const Dims& d, T* f1, const T* f2, int iplane, int opt) {
    int ighost = 0;
    if (iplane == 1) ighost = 0;
    else if (iplane == d.nx) ighost = d.nx + 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j)
            for (int l = 0; l < d.nl; ++l) {
                if ((iplane == 1 && L.cx[l] < 0) || (iplane == d.nx && L.cx[l] > 0)) {
                    int m = find_dir(L, -L.cx[l], opt * L.cy[l], opt * L.cz[l]);
                    if (m >= 0) {
                        f1[d.f(m, ighost, j, k)] = f2[d.f(l, ighost, j, k)];
                        f1[d.f(l, ighost, j, k)] = f1[d.f(l, iplane, j - L.cy[l], k - L.cz[l])];
                    }
                }
            }
}
// m_boundary_j_closed_kernel.F90:35-46
template <typename T>
void bnd_j_closed(const Lattice<T>& L, const Dims& d, T* f1, const T* f2, int jplane, int opt) {
    int jghost = 0;
    if (jplane == 1) jghost = 0;
    else if (jplane == d.ny) jghost = d.ny + 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int i = 1; i <= d.nx; ++i)
            for (int l = 0; l < d.nl; ++l) {
                if ((jplane == 1 && L.cy[l] < 0) || (jplane == d.ny && L.cy[l] > 0)) {
                    int m = find_dir(L, opt * L.cx[l], -L.cy[l], opt * L.cz[l]);
                    if (m >= 0) {
                        f1[d.f(m, i, jghost, k)] = f2[d.f(l, i, jghost, k)];
                        f1[d.f(l, i, jghost, k)] = f1[d.f(l, i - L.cx[l], jplane, k - L.cz[l])];
                    }
                }
            }
}
// m_boundary_k_closed_kernel.F90:24-46
template <typename T>
void bnd_k_closed(const Lattice<T>& L, const Dims& d, T* f1, const T* f2, int kplane, int opt) {
    int kghost = 0;
    if (kplane == 1) kghost = 0;
    else if (kplane == d.nz) kghost = d.nz + 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= d.ny; ++j)
        for (int i = 1; i <= d.nx; ++i)
            for (int l = 0; l < d.nl; ++l) {
                if ((kplane == 1 && L.cz[l] < 0) || (kplane == d.nz && L.cz[l] > 0)) {
                    int m = find_dir(L, opt * L.cx[l], opt * L.cy[l], -L.cz[l]);
                    if (m >= 0) {
                        f1[d.f(m, i, j, kghost)] = f2[d.f(l, i, j, kghost)];
                        f1[d.f(l, i, j, kghost)] = f1[d.f(l, i - L.cx[l], j - L.cy[l], kplane)];
                    }
                }
            }
}

// m_boundary_j_k_edges.F90:25-149.  Note the (ny+1,nz+1) edge's mirror keeps
// cx unchanged regardless of opt (:129), unlike the other three edges.
template <typename T>
void bnd_j_k_edges(const Lattice<T>& L, const Dims& d, T* f1, const T* f2, int opt) {
    struct E { int jg, kg, sy, sz, ji, ki, xsign_uses_opt; };
    const E edges[4] = {{0, 0, -1, -1, 1, 1, 1},
                        {d.ny + 1, 0, 1, -1, d.ny, 1, 1},
                        {0, d.nz + 1, -1, 1, 1, d.nz, 1},
                        {d.ny + 1, d.nz + 1, 1, 1, d.ny, d.nz, 0}};
    for (const E& e : edges) {
        for (int i = 1; i <= d.nx; ++i)
            for (int l = 0; l < d.nl; ++l)
                if (L.cy[l] * e.sy > 0 && L.cz[l] * e.sz > 0) {
                    int mx = e.xsign_uses_opt ? opt * L.cx[l] : L.cx[l];
                    int m = find_dir(L, mx, -L.cy[l], -L.cz[l]);
                    if (m >= 0) f1[d.f(m, i, e.jg, e.kg)] = f2[d.f(l, i, e.jg, e.kg)];
                }
        for (int i = 1; i <= d.nx; ++i)
            for (int l = 0; l < d.nl; ++l)
                if (L.cy[l] * e.sy > 0 && L.cz[l] * e.sz > 0)
                    f1[d.f(l, i, e.jg, e.kg)] = f1[d.f(l, i, e.ji, e.ki)];
    }
}
// m_boundary_i_j_edges.F90:25-145
template <typename T>
void bnd_i_j_edges(const Lattice<T>& L, const Dims& d, T* f1, const T* f2, int opt) {
    struct E { int ig, jg, sx, sy, ii, ji; };
    const E edges[4] = {{0, 0, -1, -1, 1, 1},
                        {d.nx + 1, 0, 1, -1, d.nx, 1},
                        {0, d.ny + 1, -1, 1, 1, d.ny},
                        {d.nx + 1, d.ny + 1, 1, 1, d.nx, d.ny}};
    for (const E& e : edges) {
        for (int k = 1; k <= d.nz; ++k)
            for (int l = 0; l < d.nl; ++l)
                if (L.cx[l] * e.sx > 0 && L.cy[l] * e.sy > 0) {
                    int m = find_dir(L, -L.cx[l], -L.cy[l], opt * L.cz[l]);
                    if (m >= 0) f1[d.f(m, e.ig, e.jg, k)] = f2[d.f(l, e.ig, e.jg, k)];
                }
        for (int k = 1; k <= d.nz; ++k)
            for (int l = 0; l < d.nl; ++l)
                if (L.cx[l] * e.sx > 0 && L.cy[l] * e.sy > 0)
                    f1[d.f(l, e.ig, e.jg, k)] = f1[d.f(l, e.ii, e.ji, k)];
    }
}
// m_boundary_i_k_edges.F90:3-152
template <typename T>
void bnd_i_k_edges(const Lattice<T>& L, const Dims& d, T* f1, const T* f2, int opt) {
    struct E { int ig, kg, sx, sz, ii, ki; };
    const E edges[4] = {{0, 0, -1, -1, 1, 1},
                        {d.nx + 1, 0, 1, -1, d.nx, 1},
                        {0, d.nz + 1, -1, 1, 1, d.nz},
                        {d.nx + 1, d.nz + 1, 1, 1, d.nx, d.nz}};
    for (const E& e : edges) {
        for (int j = 1; j <= d.ny; ++j)
            for (int l = 0; l < d.nl; ++l)
                if (L.cx[l] * e.sx > 0 && L.cz[l] * e.sz > 0) {
                    int m = find_dir(L, -L.cx[l], opt * L.cy[l], -L.cz[l]);
                    if (m >= 0) f1[d.f(m, e.ig, j, e.kg)] = f2[d.f(l, e.ig, j, e.kg)];
                }
        for (int j = 1; j <= d.ny; ++j)
            for (int l = 0; l < d.nl; ++l)
                if (L.cx[l] * e.sx > 0 && L.cz[l] * e.sz > 0)
                    f1[d.f(l, e.ig, j, e.kg)] = f1[d.f(l, e.ii, j, e.ki)];
    }
}
// m_boundary_closed_corners.F90:3-101
template <typename T>
void bnd_closed_corners(const Lattice<T>& L, const Dims& d, T* f1, const T* f2, int opt) {
    const int corner[8][3] = {{0, 0, 0}, {0, 0, d.nz + 1}, {0, d.ny + 1, 0}, {0, d.ny + 1, d.nz + 1},
                              {d.nx + 1, 0, 0}, {d.nx + 1, 0, d.nz + 1}, {d.nx + 1, d.ny + 1, 0},
                              {d.nx + 1, d.ny + 1, d.nz + 1}};
    for (int m = 0; m < 8; ++m) {
        int ic = corner[m][0], jc = corner[m][1], kc = corner[m][2];
        auto out = [&](int l) {
            return ((ic == 0 && L.cx[l] < 0) || (ic == d.nx + 1 && L.cx[l] > 0)) &&
                   ((jc == 0 && L.cy[l] < 0) || (jc == d.ny + 1 && L.cy[l] > 0)) &&
                   ((kc == 0 && L.cz[l] < 0) || (kc == d.nz + 1 && L.cz[l] > 0));
        };
        for (int l = 0; l < d.nl; ++l)
            if (out(l)) {
                int mm = find_dir(L, opt * L.cx[l], opt * L.cy[l], opt * L.cz[l]);
                if (mm >= 0) f1[d.f(mm, ic, jc, kc)] = f2[d.f(l, ic, jc, kc)];
            }
        for (int l = 0; l < d.nl; ++l)
            if (out(l)) f1[d.f(l, ic, jc, kc)] = f1[d.f(l, ic - L.cx[l], jc - L.cy[l], kc - L.cz[l])];
    }
}

// m_boundary_i_inflow_kernel.F90:56-111 (taperj = taperk = 1, m_boundarycond.F90:334-335)
template <typename T>
void bnd_i_inflow(const orc_params* p, const Lattice<T>& L, const Dims& d, T* f, const T* uvel) {
    const T pi = T(3.1415927410125732);
    const T rho0 = T(p->rho0);
    const T udir = T(p->udir);
    const T one = T(1.0);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j) {
            T fghost[27];
            int ka = std::min(std::max(k, 1), d.nz);
            T uu = uvel[ka - 1] * one * one;
            for (int l = 0; l < d.nl; ++l) {
                T wl = L.w[l];
                T cxl = T(L.cx[l]);
                T cyl = T(L.cy[l]);
                fghost[l] = f[d.f(l, 1, j, k)] - T(2.0) * wl * rho0 *
                            (cxl * uu * std::cos(udir * pi / T(180.0)) + cyl * uu * std::sin(udir * pi / T(180.0))) / L.cs2;
            }
            for (int l = 0; l < d.nl; ++l) {
                if (L.cx[l] <= 0) {
                    f[d.f(l, 0, j, k)] = fghost[l];
                } else {
                    int m = find_dir(L, -L.cx[l], -L.cy[l], -L.cz[l]);
                    if (m >= 0) f[d.f(l, 0, j, k)] = fghost[m];
                }
            }
            for (int l = 0; l < d.nl; ++l) f[d.f(l, d.nx + 1, j, k)] = f[d.f(l, d.nx, j, k)];
        }
}

inline void opts(int code, int& o1, int& oN) {
    switch (code) {
        case 11: o1 = -1; oN = -1; break;
        case 12: o1 = -1; oN = +1; break;
        case 21: o1 = +1; oN = -1; break;
        case 22: o1 = +1; oN = +1; break;
        default: o1 = 0; oN = 0;
    }
}

// boundarycond, m_boundarycond.F90:14-468 (dispatch order preserved)
template <typename T>
void boundarycond(const orc_params* p, T* f1, T* f2, const T* uvel) {
    const Lattice<T> L(p->nl);
    const Dims d(p);
    if (p->ibnd == 0) bnd_i_periodic(d, f1);
    if (p->jbnd == 0) bnd_j_periodic(d, f1);
    if (p->kbnd == 0) bnd_k_periodic(d, f1);
    int o1, oN;
    opts(p->ibnd, o1, oN);
    if (o1 != 0) { bnd_i_closed(L, d, f1, f2, 1, o1); bnd_i_closed(L, d, f1, f2, d.nx, oN); }
    opts(p->jbnd, o1, oN);
    if (o1 != 0) { bnd_j_closed(L, d, f1, f2, 1, o1); bnd_j_closed(L, d, f1, f2, d.ny, oN); }
    opts(p->kbnd, o1, oN);
    if (o1 != 0) { bnd_k_closed(L, d, f1, f2, 1, o1); bnd_k_closed(L, d, f1, f2, d.nz, oN); }
    if (p->jbnd > 10 && p->kbnd > 10) bnd_j_k_edges(L, d, f1, f2, (p->jbnd == 22 && p->kbnd == 22) ? 1 : -1);
    if (p->ibnd > 10 && p->jbnd > 10) bnd_i_j_edges(L, d, f1, f2, (p->ibnd == 22 && p->jbnd == 22) ? 1 : -1);
    if (p->ibnd > 10 && p->kbnd > 10) bnd_i_k_edges(L, d, f1, f2, (p->ibnd == 22 && p->kbnd == 22) ? 1 : -1);
    if (p->ibnd > 10 && p->jbnd > 10 && p->kbnd > 10) bnd_closed_corners(L, d, f1, f2, -1);
    if (p->ibnd == 1) bnd_i_inflow(p, L, d, f1, uvel);
    if (p->ibnd == 0) bnd_i_periodic(d, f1);
    if (p->jbnd == 0) bnd_j_periodic(d, f1);
    if (p->kbnd == 0) bnd_k_periodic(d, f1);
}

// solids, m_solids.F90:24-36: swap pairs (l,l+1), l=2,4,...,nl-1 (1-based)
template <typename T>
void solids(const orc_params* p, T* f, const int32_t* blanking) {
    const Dims d(p);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j)
            for (int i = 1; i <= d.nx; ++i)
                if (blanking[d.s(i, j, k)] != 0)
                    for (int l = 1; l + 1 < d.nl; l += 2) std::swap(f[d.f(l, i, j, k)], f[d.f(l + 1, i, j, k)]);
}

// fequil3_block_kernel arithmetic for one cell, m_fequil3_block_kernel.F90:62-107
template <typename T>
void feq_block_cell(const orc_params* p, const Lattice<T>& L, T rr, const T vel[3], T* out) {
    const T ratio = L.inv6cs6 / L.inv2cs4;
    T A2[3][3], A3[3][3][3];
    for (int q = 0; q < 3; ++q)
        for (int pp = 0; pp < 3; ++pp) A2[q][pp] = rr * vel[pp] * vel[q] * L.inv2cs4;
    if (p->ibgk == 3)
        for (int r = 0; r < 3; ++r) {
            T vratio = vel[r] * ratio;
            for (int q = 0; q < 3; ++q)
                for (int pp = 0; pp < 3; ++pp) A3[r][q][pp] = A2[q][pp] * vratio;
        }
    for (int l = 0; l < L.nl; ++l) {
        T cu = T(L.cx[l]) * vel[0] + T(L.cy[l]) * vel[1] + T(L.cz[l]) * vel[2];
        T tmp1 = rr * (T(1.0) + cu * L.inv1cs2);
        T tmp2 = T(0.0);
        for (int q = 0; q < 3; ++q)
            for (int pp = 0; pp < 3; ++pp) tmp2 = tmp2 + L.H2[l][q][pp] * A2[q][pp];
        T tmp3 = T(0.0);
        if (p->ibgk == 3)
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q)
                    for (int pp = 0; pp < 3; ++pp) tmp3 = tmp3 + L.H3[l][r][q][pp] * A3[r][q][pp];
        out[l] = L.w[l] * (tmp1 + tmp2 + tmp3);
    }
}

// inflow_turbulence_forcing, m_inflow_turbulence_forcing.F90:44-128
// df(nl,ny,nz); uu/vv/ww(ny,nz,0:nrturb)
template <typename T>
void turbulence_forcing(const orc_params* p, T* df, const T* rho, const T* u, const T* v, const T* w,
                        const T* uu, const T* vv, const T* ww, int it) {
    const Lattice<T> L(p->nl);
    const Dims d(p);
    const int ip = p->iturb_pos;
    int lit = it % p->nrturb;
    if (lit == 0) lit = p->nrturb;
    const T ampl = T(p->ampl);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j) {
            long c = d.s(ip, j, k);
            T rr = rho[c];
            T vel[3] = {u[c], v[c], w[c]};
            T feq1[27], feq2[27];
            feq_block_cell(p, L, rr, vel, feq1);
            long t = (long)(j - 1) + (long)d.ny * ((long)(k - 1) + (long)d.nz * lit);
            vel[0] = vel[0] + ampl * uu[t];
            vel[1] = vel[1] + ampl * vv[t];
            vel[2] = vel[2] + ampl * ww[t];
            feq_block_cell(p, L, rr, vel, feq2);
            for (int l = 0; l < d.nl; ++l)
                df[l + (long)d.nl * ((j - 1) + (long)d.ny * (k - 1))] = feq2[l] - feq1[l];
        }
}

// inflow_turbulence_apply, m_inflow_turbulence_apply.F90:19-28
template <typename T>
void turbulence_apply(const orc_params* p, T* f, const T* df) {
    const Dims d(p);
    const int ip = p->iturb_pos;
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j)
            for (int l = 0; l < d.nl; ++l)
                f[d.f(l, ip, j, k)] = f[d.f(l, ip, j, k)] + df[l + (long)d.nl * ((j - 1) + (long)d.ny * (k - 1))];
}

// forcings_apply, m_forcings_apply_kernel.F90:47-213: at interior cells with
// rho > 0, f += feq2(rho, u - F/rho) - feq2(rho, u), second-order equilibria
// (the third-order terms are commented out in the reference).  F(3,0:nx+1,0:ny+1,0:nz+1).
template <typename T>
void forcings_apply(const orc_params* p, T* f, const T* F, const T* rho, const T* u, const T* v, const T* w) {
    const Dims d(p);
    const Lattice<T> L(d.nl);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d.nz; ++k)
        for (int j = 1; j <= d.ny; ++j)
            for (int i = 1; i <= d.nx; ++i) {
                const long c = d.s(i, j, k);
                const T rr = rho[c];
                if (rr <= T(0.0)) continue;
                const T vel0[3] = {u[c], v[c], w[c]};
                const T du = -F[3 * c] / rr, dv = -F[3 * c + 1] / rr, dw = -F[3 * c + 2] / rr;
                const T vel1[3] = {vel0[0] + du, vel0[1] + dv, vel0[2] + dw};
                T A0[3][3], A1[3][3];
                for (int q = 0; q < 3; ++q)
                    for (int pp = 0; pp < 3; ++pp) {
                        A0[q][pp] = rr * vel0[pp] * vel0[q] * L.inv2cs4;
                        A1[q][pp] = rr * vel1[pp] * vel1[q] * L.inv2cs4;
                    }
                for (int l = 0; l < d.nl; ++l) {
                    T cu = T(L.cx[l]) * vel0[0] + T(L.cy[l]) * vel0[1] + T(L.cz[l]) * vel0[2];
                    T tmp1 = rr * (T(1.0) + cu * L.inv1cs2);
                    T tmp2 = T(0.0);
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) tmp2 = tmp2 + L.H2[l][q][pp] * A0[q][pp];
                    const T feq0 = L.w[l] * (tmp1 + tmp2 + T(0.0));
                    cu = T(L.cx[l]) * vel1[0] + T(L.cy[l]) * vel1[1] + T(L.cz[l]) * vel1[2];
                    tmp1 = rr * (T(1.0) + cu * L.inv1cs2);
                    tmp2 = T(0.0);
                    for (int q = 0; q < 3; ++q)
                        for (int pp = 0; pp < 3; ++pp) tmp2 = tmp2 + L.H2[l][q][pp] * A1[q][pp];
                    const T feq1 = L.w[l] * (tmp1 + tmp2 + T(0.0));
                    f[d.f(l, i, j, k)] = f[d.f(l, i, j, k)] + (feq1 - feq0);
                }
            }
}

// fillghosts, m_fillghosts.F90:18-29
template <typename T>
void fillghosts(const orc_params* p, T* f) {
    const Dims d(p);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k <= d.nz + 1; ++k)
        for (int j = 0; j <= d.ny + 1; ++j)
            for (int i = 0; i <= d.nx + 1; ++i) {
                int i1 = std::min(std::max(i, 1), d.nx);
                int j1 = std::min(std::max(j, 1), d.ny);
                int k1 = std::min(std::max(k, 1), d.nz);
                if (i1 == i && j1 == j && k1 == k) continue;
                for (int l = 0; l < d.nl; ++l) f[d.f(l, i, j, k)] = f[d.f(l, i1, j1, k1)];
            }
}

// Initialisation order of main.F90:243-247
template <typename T>
void init(const orc_params* p, T* fA, T* fB, const T* rho, const T* u, const T* v, const T* w, const T* uvel) {
    const Dims d(p);
    long n = d.ncell() * d.nl;
    std::fill(fB, fB + n, T(0.0));
    fequil3(p, fB, rho, u, v, w);
    fillghosts(p, fB);
    std::memcpy(fA, fB, sizeof(T) * n);
    boundarycond(p, fB, fA, uvel);
    boundarycond(p, fA, fB, uvel);
}

// Time loop of main.F90:283-329 (turbines, buoyancy, tracers, diagnostics off).
// On return fA holds f1 and fB holds f2 of the reference after the last step.
template <typename T>
void run(const orc_params* p, T* fA, T* fB, T* rho, T* u, T* v, T* w, T* tau, const T* ablvisc,
         const int32_t* blanking, const T* uvel, const T* uu, const T* vv, const T* ww, int it0, int nsteps,
         const T* force = nullptr) {
    const Dims d(p);
    T* f1 = fA;
    T* f2 = fB;
    std::vector<T> df;
    if (p->lturb) df.assign((size_t)d.nl * d.ny * d.nz, T(0.0));
    for (int it = it0 + 1; it <= it0 + nsteps; ++it) {
        if (p->lturb) turbulence_forcing(p, df.data(), rho, u, v, w, uu, vv, ww, it);
        postcoll(p, f1, tau, rho, u, v, w, ablvisc);
        if (p->lturb) turbulence_apply(p, f1, df.data());
        if (force) forcings_apply(p, f1, force, rho, u, v, w);   // main.F90:306
        if (p->lsolids) solids(p, f1, blanking);
        boundarycond(p, f1, f2, uvel);
        drift(p, f2, f1);
        std::swap(f1, f2);
        macrovars(p, rho, u, v, w, f1);
    }
    if (f1 != fA) {
        // odd step count: exchange the contents in place (no temporary of the state's size)
        const long n = d.ncell() * d.nl;
#pragma omp parallel for schedule(static)
        for (long e = 0; e < n; ++e) std::swap(fA[e], fB[e]);
    }
}

template <typename T>
int tables(int nl, T* H2, T* H3, T* w, int32_t* cx, int32_t* cy, int32_t* cz, int32_t* bounce) {
    if (nl != 19 && nl != 27) return -1;
    const Lattice<T> L(nl);
    for (int l = 0; l < nl; ++l) {
        w[l] = L.w[l]; cx[l] = L.cx[l]; cy[l] = L.cy[l]; cz[l] = L.cz[l]; bounce[l] = L.bounce[l];
        for (int q = 0; q < 3; ++q)
            for (int pp = 0; pp < 3; ++pp) {
                H2[pp + 3 * (q + 3 * l)] = L.H2[l][q][pp];
                for (int r = 0; r < 3; ++r) H3[pp + 3 * (q + 3 * (r + 3 * l))] = L.H3[l][r][q][pp];
            }
    }
    return 0;
}

}  // namespace

extern "C" {

void orc_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}

int orc_tables_f32(int nl, float* H2, float* H3, float* w, int32_t* cx, int32_t* cy, int32_t* cz, int32_t* b) {
    return tables<float>(nl, H2, H3, w, cx, cy, cz, b);
}
int orc_tables_f64(int nl, double* H2, double* H3, double* w, int32_t* cx, int32_t* cy, int32_t* cz, int32_t* b) {
    return tables<double>(nl, H2, H3, w, cx, cy, cz, b);
}

#define ORC_DEF(T, S)                                                                                          \
void orc_fequil3_##S(const orc_params* p, T* feq, const T* rho, const T* u, const T* v, const T* w) {          \
    fequil3<T>(p, feq, rho, u, v, w); }                                                                         \
void orc_postcoll_##S(const orc_params* p, T* f, T* tau, const T* rho, const T* u, const T* v, const T* w,    \
                      const T* ablvisc) { postcoll<T>(p, f, tau, rho, u, v, w, ablvisc); }                      \
void orc_drift_##S(const orc_params* p, T* f, const T* feq) { drift<T>(p, f, feq); }                          \
void orc_macrovars_##S(const orc_params* p, T* rho, T* u, T* v, T* w, const T* f) {                           \
    macrovars<T>(p, rho, u, v, w, f); }                                                                         \
void orc_regularization_##S(const orc_params* p, T* f, const T* feq, const T* u, const T* v, const T* w) {    \
    regularization<T>(p, f, feq, u, v, w); }                                                                    \
void orc_vreman_##S(const orc_params* p, const T* f, T* tau) { vreman<T>(p, f, tau); }                        \
void orc_compute_fneq_##S(const orc_params* p, T* f, const T* feq) { compute_fneq<T>(p, f, feq); }            \
void orc_compute_f_##S(const orc_params* p, T* f, const T* feq) { compute_f<T>(p, f, feq); }                  \
void orc_boundarycond_##S(const orc_params* p, T* f1, T* f2, const T* uvel) {                                 \
    boundarycond<T>(p, f1, f2, uvel); }                                                                         \
void orc_solids_##S(const orc_params* p, T* f, const int32_t* blanking) { solids<T>(p, f, blanking); }        \
void orc_turbulence_forcing_##S(const orc_params* p, T* df, const T* rho, const T* u, const T* v, const T* w, \
                                const T* uu, const T* vv, const T* ww, int it) {                               \
    turbulence_forcing<T>(p, df, rho, u, v, w, uu, vv, ww, it); }                                              \
void orc_turbulence_apply_##S(const orc_params* p, T* f, const T* df) { turbulence_apply<T>(p, f, df); }      \
void orc_fillghosts_##S(const orc_params* p, T* f) { fillghosts<T>(p, f); }                                   \
void orc_init_##S(const orc_params* p, T* fA, T* fB, const T* rho, const T* u, const T* v, const T* w,        \
                  const T* uvel) { init<T>(p, fA, fB, rho, u, v, w, uvel); }                                   \
void orc_run_##S(const orc_params* p, T* fA, T* fB, T* rho, T* u, T* v, T* w, T* tau, const T* ablvisc,       \
                 const int32_t* blanking, const T* uvel, const T* uu, const T* vv, const T* ww, int it0,       \
                 int nsteps) {                                                                                  \
    run<T>(p, fA, fB, rho, u, v, w, tau, ablvisc, blanking, uvel, uu, vv, ww, it0, nsteps); }                  \
void orc_run_forced_##S(const orc_params* p, T* fA, T* fB, T* rho, T* u, T* v, T* w, T* tau, const T* ablvisc,\
                        const int32_t* blanking, const T* uvel, const T* uu, const T* vv, const T* ww, int it0,\
                        int nsteps, const T* force) {                                                          \
    run<T>(p, fA, fB, rho, u, v, w, tau, ablvisc, blanking, uvel, uu, vv, ww, it0, nsteps, force); }           \
void orc_forcings_apply_##S(const orc_params* p, T* f, const T* force, const T* rho, const T* u, const T* v,   \
                            const T* w) { forcings_apply<T>(p, f, force, rho, u, v, w); }

ORC_DEF(float, f32)
ORC_DEF(double, f64)
#undef ORC_DEF

}  // extern "C"
