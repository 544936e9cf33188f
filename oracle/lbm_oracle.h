/*
 * lbm_oracle.h -- C interface of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle is a plain C++ restatement of the geirev/LBM per-timestep path
 * (Fortran 90 / CUDA Fortran, built with nvfortran or gfortran).  It exists
 * so that tests and the smoke check can compare the CUDA library against the
 * reference's arithmetic, and so that the benchmark's CPU legs (the CPU
 * baseline and the reference arm) can time it.  Nothing
 * in the product library links, loads or calls it.
 *
 * Parity status: UNPINNED against reference outputs.  The reference ships no
 * golden vectors and cannot be built in this image (no Fortran compiler), so
 * the restatement is pinned by analytic known answers (lattice identities,
 * moment conservation, equilibrium fixed points, permutation/involution
 * properties) and by a second, independent numpy restatement on small grids.
 *
 * Layout follows the reference exactly: f(nl, 0:nx+1, 0:ny+1, 0:nz+1) in
 * Fortran column-major order (l fastest), scalars (0:nx+1, 0:ny+1, 0:nz+1),
 * uvel(nz), ablvisc(nz), uu/vv/ww(ny, nz, 0:nrturb), blanking as logical(4).
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
    int32_t nx, ny, nz;          /* interior grid (mod_dimensions.F90) */
    int32_t nl;                  /* 19 (D3Q19) or 27 (D3Q27) */
    int32_t ibgk;                /* 2 or 3: order of the Hermite equilibrium */
    int32_t ihrr;                /* 1: regularized R(fneq) */
    int32_t ivreman;             /* 1: Vreman eddy viscosity */
    int32_t ibnd, jbnd, kbnd;    /* boundary codes (m_readinfile.F90:12-14) */
    int32_t iturb_pos;           /* i index of the turbulence slice (10) */
    int32_t lsolids;             /* apply solids() in the step */
    int32_t lturb;               /* inflowturbulence */
    int32_t nrturb;              /* number of turbulence fields */
    double kinevisc;             /* lattice kinematic viscosity */
    double smagorinsky;          /* Vreman/Smagorinsky constant */
    double rho0;                 /* reference density (1.0) */
    double udir;                 /* inflow direction, degrees */
    double ampl;                 /* turbulence amplitude */
} orc_params;

void orc_set_threads(int n);

/* lattice tables: H2(3,3,nl), H3(3,3,3,nl) column-major, weights(nl), c*(nl), bounce(nl) */
int orc_tables_f32(int nl, float* H2, float* H3, float* w, int32_t* cx, int32_t* cy, int32_t* cz, int32_t* bounce);
int orc_tables_f64(int nl, double* H2, double* H3, double* w, int32_t* cx, int32_t* cy, int32_t* cz, int32_t* bounce);

#define ORC_DECL(T, S) \
void orc_fequil3_##S(const orc_params* p, T* feq, const T* rho, const T* u, const T* v, const T* w); \
void orc_postcoll_##S(const orc_params* p, T* f, T* tau, const T* rho, const T* u, const T* v, const T* w, const T* ablvisc); \
void orc_drift_##S(const orc_params* p, T* f, const T* feq); \
void orc_macrovars_##S(const orc_params* p, T* rho, T* u, T* v, T* w, const T* f); \
void orc_regularization_##S(const orc_params* p, T* f, const T* feq, const T* u, const T* v, const T* w); \
void orc_vreman_##S(const orc_params* p, const T* f, T* tau); \
void orc_compute_fneq_##S(const orc_params* p, T* f, const T* feq); \
void orc_compute_f_##S(const orc_params* p, T* f, const T* feq); \
void orc_boundarycond_##S(const orc_params* p, T* f1, T* f2, const T* uvel); \
void orc_solids_##S(const orc_params* p, T* f, const int32_t* blanking); \
void orc_turbulence_forcing_##S(const orc_params* p, T* df, const T* rho, const T* u, const T* v, const T* w, \
                                const T* uu, const T* vv, const T* ww, int it); \
void orc_turbulence_apply_##S(const orc_params* p, T* f, const T* df); \
void orc_fillghosts_##S(const orc_params* p, T* f); \
void orc_init_##S(const orc_params* p, T* fA, T* fB, const T* rho, const T* u, const T* v, const T* w, const T* uvel); \
void orc_run_##S(const orc_params* p, T* fA, T* fB, T* rho, T* u, T* v, T* w, T* tau, const T* ablvisc, \
                 const int32_t* blanking, const T* uvel, const T* uu, const T* vv, const T* ww, int it0, int nsteps); \
void orc_run_forced_##S(const orc_params* p, T* fA, T* fB, T* rho, T* u, T* v, T* w, T* tau, const T* ablvisc, \
                        const int32_t* blanking, const T* uvel, const T* uu, const T* vv, const T* ww, int it0, \
                        int nsteps, const T* force); \
void orc_forcings_apply_##S(const orc_params* p, T* f, const T* force, const T* rho, const T* u, const T* v, \
                            const T* w);

ORC_DECL(float, f32)
ORC_DECL(double, f64)
#undef ORC_DECL

#ifdef __cplusplus
}
#endif
#endif
