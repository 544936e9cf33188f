// api.cu -- C ABI of the B200 LBM library (declarations in include/lbm_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/lbm_b200.h"
#include "boundary.cuh"
#include "ref_kernels.cuh"
#include "state_kernels.cuh"
#include "pair_step.cuh"

using namespace lbm;

// ---------------------------------------------------------------------------
// Scratch of lbm_mass_momentum_noalloc: a fixed device array instead of a
// cudaMalloc'ed buffer.  LBM_NOALLOC_BLOCKS block partials of 4 doubles
// (64 KiB), one block per LBM_NOALLOC_CHUNK interior cells, so grids of up to
// 2048 * 65536 = 134,217,728 interior cells.  Every GPU that loads the library
// holds this array until the process exits.
// ---------------------------------------------------------------------------
#define LBM_NOALLOC_BLOCKS 2048
#define LBM_NOALLOC_CHUNK 65536LL
static __device__ __align__(256) double g_noalloc_partial[LBM_NOALLOC_BLOCKS * 4];

enum { ST_NONE = 0, ST_PRE = 1, ST_POST = 2 };
// blocks of the conservation reduction (a few per SM)
#define LBM_SUM_BLOCKS 1184

struct lbm_ctx {
    lbm_params p;
    int dev = 0;
    cudaStream_t stream = nullptr;   // legacy default stream unless lbm_set_stream gives another
    std::string err;
    RefGrid rg;
    SoaGrid sg;
    CollideParams cp;
    CollideParamsT<double> cpd;      // the FP64 entry points' parameters (the reference's DP build)
    double rho0d = 1.0, cosdd = 1.0, sindd = 0.0;
    FacePairs face[3][2];
    bool face_on[3] = {false, false, false};
    EdgeSet edges[3];
    bool edges_on[3] = {false, false, false};
    CornerSet corners;
    bool corners_on = false;
    float cosd = 1.f, sind = 0.f;
    // fused state
    void* buf[2] = {nullptr, nullptr};   // the two buffers a step reads and writes
    void* own[2] = {nullptr, nullptr};   // the context's allocations (buf may point at a caller's, lbm_step_to)
    size_t elem = 4;
    int cur = 0;
    int state = ST_NONE;
    float* d_macro = nullptr;     // rho,u,v,w (4 x ghost-inclusive grid) of an imported state
    uint8_t* d_solid = nullptr;   // interior solid mask
    float* d_turb = nullptr;      // uu,vv,ww copies
    int nrturb = 0;
    float ampl = 0.f;
    bool fold = false;            // boundaries folded into the step kernel (see state_kernels.cuh)
    bool fold_cfg = false;        // the boundary codes allow folding (fold unless halo_j)
    bool halo_j = false;          // j ghost planes filled by the caller's halo exchange (lbm_set_halo_j)
    void* d_edge = nullptr;       // populations at i=1 and i=nx of the latest step
    void* d_xg[2] = {nullptr, nullptr};  // compact x-ghost columns of each buffer (folded boundaries)
    bool idx32 = true;            // state small enough for 32-bit element offsets (k_step_fast)
    int kernel = LBM_KERNEL_PAIR; // steady step kernel (lbm_set_kernel); PULL where PAIR does not apply
    int nsm = 148;
    int kopt_lo = 0, kopt_hi = 0;
    float* d_uvel = nullptr;      // uvel(nz)
    const float* force = nullptr; // caller's external_forcing(3,0:nx+1,0:ny+1,0:nz+1), read every step (lbm_set_forcing)
    float* d_abl = nullptr;       // ablvisc(nz), zero unless set
    int* d_it = nullptr;          // number of the step being computed
    int* d_status = nullptr;
    float* d_adj_terms = nullptr; // 4 x cells: the macrovars adjoint terms of lbm_macrovars_drift_adj (allocated on first use)
    double* d_partial = nullptr;  // FP64 block partials of the conservation sums (scratch)
    double* d_sum = nullptr;      // their total (4 doubles)
    int it = 0;
    // instrumentation: kernel launches issued, optional event timing of the step
    // kernel and of the boundary launches that follow it
    long long launches = 0;
    bool profiling = false;
    std::vector<cudaEvent_t> ev;   // triples (before the step kernel, after it, after the boundaries)
    size_t ev_used = 0;
    double prof_ms = 0.0;
    double prof_bc_ms = 0.0;
    long long prof_launches = 0;
};

namespace {

// bytes of one state buffer: nl direction blocks of dstride elements
size_t state_bytes_of(const lbm_ctx* c) { return (size_t)c->p.nl * c->sg.dstride * c->elem; }

int fail(lbm_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

int cuda_check(lbm_ctx* c, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return LBM_OK;
    return fail(c, e == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define LBM_TRY(...)                    \
    do {                                \
        int _rc = (__VA_ARGS__);        \
        if (_rc != LBM_OK) return _rc;  \
    } while (0)
// after a launch: the launch's error, which cudaGetLastError also clears (an error
// left pending by earlier work of the calling thread is reported here and cleared too)
#define LBM_LAUNCHED(c, what) LBM_TRY(cuda_check((c), cudaGetLastError(), (what)))

// accumulate the elapsed times of recorded event triples, then reuse them
int prof_drain(lbm_ctx* c) {
    if (c->ev_used == 0) return LBM_OK;
    int rc = cuda_check(c, cudaEventSynchronize(c->ev[3 * c->ev_used - 1]), "profile");
    if (rc != LBM_OK) return rc;
    for (size_t q = 0; q < c->ev_used; ++q) {
        float ms = 0.f, bc = 0.f;
        rc = cuda_check(c, cudaEventElapsedTime(&ms, c->ev[3 * q], c->ev[3 * q + 1]), "profile");
        if (rc == LBM_OK) rc = cuda_check(c, cudaEventElapsedTime(&bc, c->ev[3 * q + 1], c->ev[3 * q + 2]), "profile");
        if (rc != LBM_OK) return rc;
        c->prof_ms += ms;
        c->prof_bc_ms += bc;
    }
    c->ev_used = 0;
    return LBM_OK;
}
// before the step kernel
int prof_begin(lbm_ctx* c) {
    if (!c->profiling) return LBM_OK;
    if (c->ev_used * 3 >= c->ev.size()) LBM_TRY(prof_drain(c));
    return cuda_check(c, cudaEventRecord(c->ev[3 * c->ev_used], c->stream), "profile");
}
// after the step kernel
int prof_end(lbm_ctx* c) {
    if (!c->profiling) return LBM_OK;
    return cuda_check(c, cudaEventRecord(c->ev[3 * c->ev_used + 1], c->stream), "profile");
}
// after the step's boundary launches (none: right after prof_end)
int prof_bound(lbm_ctx* c) {
    if (!c->profiling) return LBM_OK;
    LBM_TRY(cuda_check(c, cudaEventRecord(c->ev[3 * c->ev_used + 2], c->stream), "profile"));
    c->ev_used++;
    c->prof_launches++;
    return LBM_OK;
}
#define NEED(c, ptr) \
    if ((ptr) == nullptr) return fail((c), LBM_ERR_ARG, "%s: null pointer argument '%s'", __func__, #ptr)

int lat_find(int nl, int x, int y, int z) {
    for (int m = 0; m < nl; ++m)
        if (lat_cx(m) == x && lat_cy(m) == y && lat_cz(m) == z) return m;
    return -1;
}

void closed_opts(int code, int& o1, int& oN) {
    switch (code) {
        case 11: o1 = -1; oN = -1; break;
        case 12: o1 = -1; oN = +1; break;
        case 21: o1 = +1; oN = -1; break;
        case 22: o1 = +1; oN = +1; break;
        default: o1 = 0; oN = 0;
    }
}

// outgoing directions of a closed face and their reflections, in the order and
// with the first-match rule of m_boundary_{i,j,k}_closed_kernel.F90
FacePairs face_pairs(int nl, int axis, int side, int opt) {
    FacePairs fp;
    memset(&fp, 0, sizeof(fp));
    for (int l = 0; l < nl; ++l) {
        int c[3] = {lat_cx(l), lat_cy(l), lat_cz(l)};
        if (!((side == 0 && c[axis] < 0) || (side == 1 && c[axis] > 0))) continue;
        int mv[3] = {opt * c[0], opt * c[1], opt * c[2]};
        mv[axis] = -c[axis];
        int m = lat_find(nl, mv[0], mv[1], mv[2]);
        if (m < 0) continue;
        fp.l[fp.n] = (int8_t)l;
        fp.m[fp.n] = (int8_t)m;
        fp.cx[fp.n] = (int8_t)c[0];
        fp.cy[fp.n] = (int8_t)c[1];
        fp.cz[fp.n] = (int8_t)c[2];
        fp.n++;
    }
    return fp;
}

// one edge: ghost coords g (free axis -1), outgoing sign pattern s (0 = any),
// mirror rule mr (component multipliers), pass-2 source coords src
EdgeDesc edge_desc(int nl, const int g[3], const int s[3], const int mr[3], const int src[3]) {
    EdgeDesc d;
    memset(&d, 0, sizeof(d));
    d.gi = g[0]; d.gj = g[1]; d.gk = g[2];
    d.si = src[0]; d.sj = src[1]; d.sk = src[2];
    for (int l = 0; l < nl; ++l) {
        int c[3] = {lat_cx(l), lat_cy(l), lat_cz(l)};
        bool out = true;
        for (int a = 0; a < 3; ++a)
            if (s[a] != 0 && c[a] * s[a] <= 0) out = false;
        if (!out) continue;
        int m = lat_find(nl, mr[0] * c[0], mr[1] * c[1], mr[2] * c[2]);
        if (m < 0 || d.n >= 3) continue;
        d.l[d.n] = (int8_t)l;
        d.m[d.n] = (int8_t)m;
        d.n++;
    }
    return d;
}

void setup_boundaries(lbm_ctx* c) {
    const int nl = c->p.nl, nx = c->p.nx, ny = c->p.ny, nz = c->p.nz;
    const int codes[3] = {c->p.ibnd, c->p.jbnd, c->p.kbnd};
    for (int a = 0; a < 3; ++a) {
        int o1, oN;
        closed_opts(codes[a], o1, oN);
        c->face_on[a] = (o1 != 0);
        if (c->face_on[a]) {
            c->face[a][0] = face_pairs(nl, a, 0, o1);
            c->face[a][1] = face_pairs(nl, a, 1, oN);
        }
    }
    const int ib = c->p.ibnd, jb = c->p.jbnd, kb = c->p.kbnd;
    // j-k edges (m_boundary_j_k_edges.F90): free axis i; the (ny+1,nz+1) edge keeps cx (:129)
    c->edges_on[0] = (jb > 10 && kb > 10);
    if (c->edges_on[0]) {
        const int opt = (jb == 22 && kb == 22) ? 1 : -1;
        EdgeSet& es = c->edges[0];
        es.free_axis = 0; es.nfree = nx; es.nedges = 4;
        const int G[4][3] = {{-1, 0, 0}, {-1, ny + 1, 0}, {-1, 0, nz + 1}, {-1, ny + 1, nz + 1}};
        const int S[4][3] = {{0, -1, -1}, {0, 1, -1}, {0, -1, 1}, {0, 1, 1}};
        const int SRC[4][3] = {{-1, 1, 1}, {-1, ny, 1}, {-1, 1, nz}, {-1, ny, nz}};
        for (int e = 0; e < 4; ++e) {
            const int mr[3] = {e == 3 ? 1 : opt, -1, -1};
            es.e[e] = edge_desc(nl, G[e], S[e], mr, SRC[e]);
        }
    }
    // i-j edges (m_boundary_i_j_edges.F90): free axis k
    c->edges_on[1] = (ib > 10 && jb > 10);
    if (c->edges_on[1]) {
        const int opt = (ib == 22 && jb == 22) ? 1 : -1;
        EdgeSet& es = c->edges[1];
        es.free_axis = 2; es.nfree = nz; es.nedges = 4;
        const int G[4][3] = {{0, 0, -1}, {nx + 1, 0, -1}, {0, ny + 1, -1}, {nx + 1, ny + 1, -1}};
        const int S[4][3] = {{-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 1, 0}};
        const int SRC[4][3] = {{1, 1, -1}, {nx, 1, -1}, {1, ny, -1}, {nx, ny, -1}};
        const int mr[3] = {-1, -1, opt};
        for (int e = 0; e < 4; ++e) es.e[e] = edge_desc(nl, G[e], S[e], mr, SRC[e]);
    }
    // i-k edges (m_boundary_i_k_edges.F90): free axis j
    c->edges_on[2] = (ib > 10 && kb > 10);
    if (c->edges_on[2]) {
        const int opt = (ib == 22 && kb == 22) ? 1 : -1;
        EdgeSet& es = c->edges[2];
        es.free_axis = 1; es.nfree = ny; es.nedges = 4;
        const int G[4][3] = {{0, -1, 0}, {nx + 1, -1, 0}, {0, -1, nz + 1}, {nx + 1, -1, nz + 1}};
        const int S[4][3] = {{-1, 0, -1}, {1, 0, -1}, {-1, 0, 1}, {1, 0, 1}};
        const int SRC[4][3] = {{1, -1, 1}, {nx, -1, 1}, {1, -1, nz}, {nx, -1, nz}};
        const int mr[3] = {-1, opt, -1};
        for (int e = 0; e < 4; ++e) es.e[e] = edge_desc(nl, G[e], S[e], mr, SRC[e]);
    }
    // corners (m_boundary_closed_corners.F90), always no-slip
    c->corners_on = (ib > 10 && jb > 10 && kb > 10);
    if (c->corners_on) {
        CornerSet& cs = c->corners;
        int q = 0;
        for (int ii = 0; ii < 2; ++ii)
            for (int jj = 0; jj < 2; ++jj)
                for (int kk = 0; kk < 2; ++kk, ++q) {
                    cs.ci[q] = ii ? nx + 1 : 0;
                    cs.cj[q] = jj ? ny + 1 : 0;
                    cs.ck[q] = kk ? nz + 1 : 0;
                    const int sx = ii ? 1 : -1, sy = jj ? 1 : -1, sz = kk ? 1 : -1;
                    cs.l[q] = -1;
                    cs.m[q] = -1;
                    for (int l = 0; l < nl; ++l)
                        if (lat_cx(l) * sx > 0 && lat_cy(l) * sy > 0 && lat_cz(l) * sz > 0) {
                            cs.l[q] = l;
                            cs.m[q] = lat_find(nl, -lat_cx(l), -lat_cy(l), -lat_cz(l));
                            cs.cx[q] = (int8_t)lat_cx(l);
                            cs.cy[q] = (int8_t)lat_cy(l);
                            cs.cz[q] = (int8_t)lat_cz(l);
                        }
                }
    }
    // the reference's configuration (inflow/outflow i, periodic j, closed k) runs with folded boundaries
    int ko1, koN;
    closed_opts(kb, ko1, koN);
    c->fold_cfg = (ib == 1 && jb == 0 && ko1 != 0);
    c->fold = c->fold_cfg;
    c->kopt_lo = ko1;
    c->kopt_hi = koN;
    // m_boundary_i_inflow_kernel.F90:35,71-73: cos(udir*pi/180), sin(udir*pi/180) in single precision
    const float pi = 3.1415927410125732f;
    c->cosd = cosf(c->p.udir * pi / 180.0f);
    c->sind = sinf(c->p.udir * pi / 180.0f);
}

// Parameters of the FP64 entry points, as the reference's DP build (-r8) holds
// them: every real in double precision, tiny() and eps = sqrt(tiny) of double
// (m_postcoll.F90:46-47), pi the same literal as in single precision
// (m_boundary_i_inflow_kernel.F90:35,71-73).
void set_params_f64(lbm_ctx* c, double kinevisc, double smagorinsky, double rho0, double udir) {
    c->cpd.kinevisc = kinevisc;
    c->cpd.cvre = 2.5 * smagorinsky * smagorinsky;
    c->cpd.eps = std::sqrt(lat_tiny<double>());
    c->cpd.tau0 = 3.0 * kinevisc + 0.5;
    c->cpd.ibgk = c->p.ibgk;
    c->cpd.ihrr = c->p.ihrr;
    c->cpd.ivreman = c->p.ivreman;
    c->rho0d = rho0;
    const double pi = 3.1415927410125732;
    c->cosdd = std::cos(udir * pi / 180.0);
    c->sindd = std::sin(udir * pi / 180.0);
}

// boundarycond in the dispatch order of m_boundarycond.F90:14-468
template <int Q, typename Acc>
int run_bc(lbm_ctx* c, Acc f1, Acc f2, const typename Acc::real* uvel) {
    const int nx = c->p.nx, ny = c->p.ny, nz = c->p.nz, nl = c->p.nl;
    cudaStream_t s = c->stream;
    auto periodic = [&](int axis) {
        dim3 blk(128);
        dim3 grd;
        if (axis == 0) grd = dim3((ny + 2 + 127) / 128, nz + 2, nl);
        else if (axis == 1) grd = dim3((nx + 2 + 127) / 128, nz + 2, nl);
        else grd = dim3((nx + 2 + 127) / 128, ny + 2, nl);
        k_periodic<Acc><<<grd, blk, 0, s>>>(f1, axis, nl);
        c->launches++;
    };
    const int codes[3] = {c->p.ibnd, c->p.jbnd, c->p.kbnd};
    for (int a = 0; a < 3; ++a)
        if (codes[a] == 0) periodic(a);
    for (int a = 0; a < 3; ++a) {
        if (!c->face_on[a]) continue;
        const int na = (a == 0) ? ny : nx;                  // first tangential extent
        const int nb = (a == 2) ? ny : nz;                  // second tangential extent
        dim3 grd((na + 127) / 128, nb, 2);
        k_closed<Acc><<<grd, 128, 0, s>>>(f1, f2, a, c->face[a][0], c->face[a][1], 1, 1);
        c->launches++;
    }
    for (int e = 0; e < 3; ++e) {
        if (!c->edges_on[e]) continue;
        const EdgeSet& es = c->edges[e];
        k_edges<Acc><<<dim3((es.nfree + 127) / 128, 4), 128, 0, s>>>(f1, f2, es);
        c->launches++;
    }
    if (c->corners_on) {
        k_corners<Acc><<<1, 32, 0, s>>>(f1, f2, c->corners);
        c->launches++;
    }
    if (c->p.ibnd == 1) {
        if constexpr (std::is_same<typename Acc::real, double>::value)
            k_inflow<Q, Acc><<<dim3((ny + 127) / 128, nz), 128, 0, s>>>(f1, uvel, c->rho0d, c->cosdd, c->sindd);
        else
            k_inflow<Q, Acc><<<dim3((ny + 127) / 128, nz), 128, 0, s>>>(f1, uvel, c->p.rho0, c->cosd, c->sind);
        c->launches++;
    }
    for (int a = 0; a < 3; ++a)
        if (codes[a] == 0) periodic(a);
    LBM_LAUNCHED(c, "boundarycond");
    return LBM_OK;
}

template <int Q, typename R>
int bc_ref(lbm_ctx* c, R* f1, R* f2, const R* uvel) {
    AosAccT<R> a1{f1, c->rg}, a2{f2, c->rg};
    return run_bc<Q>(c, a1, a2, uvel);
}

template <int Q, typename S>
int bc_state(lbm_ctx* c, int i1, int i2) {
    SoaAcc<S> a1{(S*)c->buf[i1], c->sg}, a2{(S*)c->buf[i2], c->sg};
    return run_bc<Q>(c, a1, a2, c->d_uvel);
}

StepArgs step_args(lbm_ctx* c) {
    StepArgs a;
    memset(&a, 0, sizeof(a));
    a.g = c->sg;
    a.cp = c->cp;
    a.solid = c->d_solid;
    if (c->nrturb > 0) {
        const long long n = (long long)c->p.ny * c->p.nz * (c->nrturb + 1);
        a.uu = c->d_turb;
        a.vv = c->d_turb + n;
        a.ww = c->d_turb + 2 * n;
    }
    a.nrturb = c->nrturb;
    a.ampl = c->ampl;
    a.iturb = c->p.iturb_pos;
    a.d_it = c->d_it;
    a.abl = c->d_abl;
    a.status = c->d_status;
    const long long g = c->rg.ncell();
    a.rho_in = c->d_macro;
    a.u_in = c->d_macro + g;
    a.v_in = c->d_macro + 2 * g;
    a.w_in = c->d_macro + 3 * g;
    a.kopt_lo = c->kopt_lo;
    a.kopt_hi = c->kopt_hi;
    a.uvel = c->d_uvel;
    a.rho0 = c->p.rho0;
    a.cosd = c->cosd;
    a.sind = c->sind;
    a.d_it_rw = c->d_it;
    a.edge = c->d_edge;
    a.full_sector = (c->p.nx % (32 / (int)c->elem)) == 0;
    a.xg_dst = c->d_xg[1 - c->cur];
    a.force = c->force;
    {
        const SoaGrid& g = c->sg;
        const long long plane = (long long)g.pitch * (g.ny + 2);
        for (int l = 0; l < c->p.nl; ++l) {
            const long long d = lat_cx(l) + (long long)lat_cy(l) * g.pitch + (long long)lat_cz(l) * plane;
            const long long po = (long long)l * g.dstride - d, so = (long long)l * g.dstride;
            a.poff[l] = (int)po;   // read only when the state fits 32-bit offsets (idx32)
            a.soff[l] = (int)so;
            a.poffb[l] = po * (long long)c->elem;
            a.soffb[l] = so * (long long)c->elem;
        }
    }
    return a;
}

template <int Q, typename S>
void launch_gather_xg(lbm_ctx* c, int b) {
    const long long n = 2LL * Q * c->sg.ny * c->sg.nz;
    k_gather_xg<Q, S><<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>((const S*)c->buf[b], (S*)c->d_xg[b], c->sg);
    c->launches++;
}

// A kernel launch that may begin while the previous kernel in the stream finishes
// (programmatic dependent launch; the kernel waits for it, see pdl_enter).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
#ifdef LBM_NO_PDL
    cfg.numAttrs = 0;
#else
    cfg.numAttrs = 1;
#endif
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

// the two-cells-per-thread kernel (pair_step.cuh) covers the regularized collision on even nx, at any
// state size (64-bit byte offsets)
bool pair_shape_ok(const lbm_ctx* c) { return c->p.ihrr == 1 && c->p.nx % 2 == 0 && c->p.nx >= 4; }
bool pair_ok(const lbm_ctx* c) { return c->kernel == LBM_KERNEL_PAIR && pair_shape_ok(c); }
dim3 pair_grid(const lbm_ctx* c, int t) { return dim3((unsigned)((c->p.nx / 2 + t - 1) / t), c->p.ny, c->p.nz); }

template <int Q, typename S, bool WRAP, bool FORCE, bool FOLD, int T>
cudaError_t pair_launch(lbm_ctx* c, const S* src, S* dst, const StepArgs& a) {
    return launch_pdl(k_step_pair<Q, S, WRAP, FORCE, FOLD, T>, pair_grid(c, T), dim3(T), c->stream, src, dst, a);
}

// the steady step from buffer cur into nxt, two cells per thread
template <int Q, typename S, bool WRAP, bool FOLD>
int pair_family_step(lbm_ctx* c, int nxt, const StepArgs& a) {
    const S* src = (const S*)c->buf[c->cur];
    S* dst = (S*)c->buf[nxt];
    // blocks of 256 threads where that shape is compiled and a row's pairs fill them
    const bool wide = pair_wide_ok<Q, S>() && (c->p.nx / 2) % 256 == 0;
    cudaError_t r;
    if (c->force)
        r = wide ? pair_launch<Q, S, WRAP, true, FOLD, pair_wide_ok<Q, S>() ? 256 : 128>(c, src, dst, a)
                 : pair_launch<Q, S, WRAP, true, FOLD, 128>(c, src, dst, a);
    else
        r = wide ? pair_launch<Q, S, WRAP, false, FOLD, pair_wide_ok<Q, S>() ? 256 : 128>(c, src, dst, a)
                 : pair_launch<Q, S, WRAP, false, FOLD, 128>(c, src, dst, a);
    LBM_TRY(cuda_check(c, r, "fused step (pair)"));
    c->launches++;
    LBM_LAUNCHED(c, "fused step (pair)");
    return LBM_OK;
}

template <int Q, typename S>
int step_one(lbm_ctx* c) {
    if (c->force && !pair_ok(c))
        return fail(c, LBM_ERR_UNSUPPORTED, "step: the fused external forcing runs in the two-cells-per-thread kernel "
                                            "(LBM_KERNEL_PAIR, ihrr = 1, even nx >= 4); use lbm_forcings_apply per call");
    const SoaGrid& g = c->sg;
    dim3 grd((g.nx + 127) / 128, g.ny, g.nz);
    StepArgs a = step_args(c);
    bool timed = false;   // a steady step of the general configuration (profile events open)
    if (c->state == ST_PRE) {
        S* b = (S*)c->buf[c->cur];
        k_step<Q, S, false, false><<<grd, 128, 0, c->stream>>>(b, b, a);
        c->launches++;
        LBM_LAUNCHED(c, "collide");
        if (c->force) {
            k_force_state<Q, S><<<grd, 128, 0, c->stream>>>(b, a);
            c->launches++;
            LBM_LAUNCHED(c, "external forcing");
        }
        c->state = ST_POST;
    } else if (c->fold) {
        const int nxt = 1 - c->cur;
        LBM_TRY(prof_begin(c));
        if (c->halo_j) {
            // a j-slab tile: pull the stored halo planes, keep the folded boundaries
            if (!pair_ok(c))
                return fail(c, LBM_ERR_UNSUPPORTED, "step: a j-slab tile in the folded configuration runs the "
                                                    "two-cells-per-thread kernel (LBM_KERNEL_PAIR, ihrr = 1, even nx >= 4)");
            LBM_TRY((pair_family_step<Q, S, false, true>(c, nxt, a)));
        } else if (pair_ok(c)) {
            LBM_TRY((pair_family_step<Q, S, true, true>(c, nxt, a)));
        } else {
            if (c->idx32)
                k_step_fast<Q, S, true><<<grd, 128, 0, c->stream>>>((const S*)c->buf[c->cur], (S*)c->buf[nxt], a);
            else
                k_step<Q, S, true, true><<<grd, 128, 0, c->stream>>>((const S*)c->buf[c->cur], (S*)c->buf[nxt], a);
            c->launches++;
            LBM_LAUNCHED(c, "fused step");
        }
        LBM_TRY(prof_end(c));
        const int nface = bc_fold_face_blocks(g);
        const int nblk = nface + (int)bc_fold_xg_blocks(g, Q, false);
        LBM_TRY(cuda_check(c, launch_pdl(k_bc_fold<Q, S>, dim3(nblk), dim3(128), c->stream, (S*)c->buf[nxt],
                                         (const S*)c->buf[c->cur], a, nface), "folded boundaries"));
        c->launches++;
        LBM_LAUNCHED(c, "folded boundaries");
        LBM_TRY(prof_bound(c));
        c->cur = nxt;
        c->it += 1;
        return LBM_OK;
    } else {
        const int nxt = 1 - c->cur;
        LBM_TRY(prof_begin(c));
        if (pair_ok(c)) {
            LBM_TRY((pair_family_step<Q, S, false, false>(c, nxt, a)));
        } else {
            if (c->idx32)
                k_step_fast<Q, S, false><<<grd, 128, 0, c->stream>>>((const S*)c->buf[c->cur], (S*)c->buf[nxt], a);
            else
                k_step<Q, S, true, false><<<grd, 128, 0, c->stream>>>((const S*)c->buf[c->cur], (S*)c->buf[nxt], a);
            c->launches++;
            LBM_LAUNCHED(c, "fused step");
        }
        LBM_TRY(prof_end(c));
        timed = true;
        c->cur = nxt;
    }
    LBM_TRY(bc_state<Q, S>(c, c->cur, 1 - c->cur));
    if (c->fold) launch_gather_xg<Q, S>(c, c->cur);
    k_bump_step<<<1, 32, 0, c->stream>>>(c->d_it);
    c->launches++;
    LBM_LAUNCHED(c, "step counter");
    if (timed) LBM_TRY(prof_bound(c));   // the boundaries of a timed step
    c->it += 1;
    return LBM_OK;
}

// dst takes the place of the buffer the next step would overwrite: it receives
// that buffer's ghost shell (the boundaries read ghost values of two steps before)
void take_dst(lbm_ctx* c, void* dst) {
    void* prev = c->buf[1 - c->cur];
    if (prev != dst) {
        if (c->fold) {
            const dim3 grd((unsigned)((fold_ghost_cells(c->sg) + 127) / 128), (unsigned)c->p.nl);
            if (c->elem == 2)
                k_copy_ghosts_fold<uint16_t><<<grd, 128, 0, c->stream>>>((uint16_t*)dst, (const uint16_t*)prev, c->sg);
            else
                k_copy_ghosts_fold<uint32_t><<<grd, 128, 0, c->stream>>>((uint32_t*)dst, (const uint32_t*)prev, c->sg);
        } else {
            const dim3 grd((unsigned)((ghost_cells(c->sg) + 127) / 128), (unsigned)c->p.nl);
            if (c->elem == 2)
                k_copy_ghosts<uint16_t><<<grd, 128, 0, c->stream>>>((uint16_t*)dst, (const uint16_t*)prev, c->sg);
            else
                k_copy_ghosts<uint32_t><<<grd, 128, 0, c->stream>>>((uint32_t*)dst, (const uint32_t*)prev, c->sg);
        }
        c->launches++;
    }
    c->buf[1 - c->cur] = dst;
}

// the next step writes into one of the context's own buffers (not the one it reads)
void own_dst(lbm_ctx* c) {
    const int n = 1 - c->cur;
    if ((c->buf[n] == c->own[0] || c->buf[n] == c->own[1]) && c->buf[n] != c->buf[c->cur]) return;
    take_dst(c, (c->buf[c->cur] == c->own[n]) ? c->own[1 - n] : c->own[n]);
}

int step_dispatch(lbm_ctx* c) {
    const bool h = c->p.storage == LBM_STORE_F16;
    if (c->p.nl == 27) return h ? step_one<27, __half>(c) : step_one<27, float>(c);
    return h ? step_one<19, __half>(c) : step_one<19, float>(c);
}

template <int Q, typename S>
void launch_import(lbm_ctx* c, const float* ref, int b) {
    const SoaGrid& g = c->sg;
    k_import<Q, S><<<dim3((g.nx + 2 + 127) / 128, g.ny + 2, g.nz + 2), 128, 0, c->stream>>>(ref, (S*)c->buf[b], g);
    c->launches++;
    if (c->fold) launch_gather_xg<Q, S>(c, b);
}
// compact x-ghost array of buffer b, or null where the rows hold the x-ghosts
template <typename S>
const S* xg_of(const lbm_ctx* c, int b) { return c->fold ? (const S*)c->d_xg[b] : nullptr; }
// after a step, periodic-j ghost rows are read as rows ny and 1 (state_kernels.cuh)
int wrap_rows(const lbm_ctx* c) { return (c->state == ST_POST && c->p.jbnd == 0 && !c->halo_j) ? 1 : 0; }

template <int Q, typename S>
void launch_export(lbm_ctx* c, float* ref, int b, bool pull) {
    const SoaGrid& g = c->sg;
    dim3 grd((g.nx + 2 + 127) / 128, g.ny + 2, g.nz + 2);
    if (pull)
        k_export<Q, S, true><<<grd, 128, 0, c->stream>>>((const S*)c->buf[b], (const S*)c->buf[1 - b], ref, g,
                                                        wrap_rows(c), xg_of<S>(c, 1 - b));
    else
        k_export<Q, S, false><<<grd, 128, 0, c->stream>>>((const S*)c->buf[b], nullptr, ref, g, wrap_rows(c),
                                                         xg_of<S>(c, b));
    c->launches++;
}
template <int Q, typename S>
void launch_macro(lbm_ctx* c, float* rho, float* u, float* v, float* w) {
    const SoaGrid& g = c->sg;
    k_macro<Q, S><<<dim3((g.nx + 2 + 127) / 128, g.ny + 2, g.nz + 2), 128, 0, c->stream>>>(
        (const S*)c->buf[c->cur], (const S*)c->buf[1 - c->cur], rho, u, v, w, g, wrap_rows(c),
        xg_of<S>(c, 1 - c->cur));
    c->launches++;
}

template <int Q, typename S>
void launch_sum_state(lbm_ctx* c) {
    k_sum_state<Q, S><<<LBM_SUM_BLOCKS, 256, 0, c->stream>>>((const S*)c->buf[c->cur], c->sg, wrap_rows(c),
                                                            c->d_partial);
    c->launches++;
}
template <int Q, typename S>
void launch_sum_pre(lbm_ctx* c) {
    k_sum_stored<Q, S><<<LBM_SUM_BLOCKS, 256, 0, c->stream>>>((const S*)c->buf[c->cur], c->sg, c->d_partial);
    c->launches++;
}

#define DISPATCH_QS(c, FN, ...)                                                        \
    do {                                                                               \
        const bool _h = (c)->p.storage == LBM_STORE_F16;                               \
        if ((c)->p.nl == 27) {                                                         \
            if (_h) FN<27, __half>(__VA_ARGS__); else FN<27, float>(__VA_ARGS__);     \
        } else {                                                                       \
            if (_h) FN<19, __half>(__VA_ARGS__); else FN<19, float>(__VA_ARGS__);     \
        }                                                                              \
    } while (0)

// ---- per-call kernels in either arithmetic type: R = float (the reference's
// default build) or double (its DP build); the entry points check arguments ----
template <typename R>
const CollideParamsT<R>& cp_of(const lbm_ctx* c);
template <>
const CollideParamsT<float>& cp_of<float>(const lbm_ctx* c) { return c->cp; }
template <>
const CollideParamsT<double>& cp_of<double>(const lbm_ctx* c) { return c->cpd; }

dim3 interior_rows(const lbm_ctx* c) { return dim3((c->p.nx + 127) / 128, c->p.ny, c->p.nz); }

template <typename R>
int fequil3_run(lbm_ctx* c, R* feq, const R* rho, const R* u, const R* v, const R* w) {
    if (c->p.nl == 27) k_ref_fequil3<27, R><<<interior_rows(c), 128, 0, c->stream>>>(feq, rho, u, v, w, c->rg, c->p.ibgk);
    else k_ref_fequil3<19, R><<<interior_rows(c), 128, 0, c->stream>>>(feq, rho, u, v, w, c->rg, c->p.ibgk);
    c->launches++;
    LBM_LAUNCHED(c, "fequil3");
    return LBM_OK;
}

template <typename R>
int postcoll_run(lbm_ctx* c, R* f, R* tau, const R* rho, const R* u, const R* v, const R* w, const R* ablvisc) {
    const CollideParamsT<R>& cp = cp_of<R>(c);
    if (c->p.nl == 27) k_ref_postcoll<27, R><<<interior_rows(c), 128, 0, c->stream>>>(f, tau, rho, u, v, w, ablvisc, c->rg, cp);
    else k_ref_postcoll<19, R><<<interior_rows(c), 128, 0, c->stream>>>(f, tau, rho, u, v, w, ablvisc, c->rg, cp);
    c->launches++;
    LBM_LAUNCHED(c, "postcoll");
    return LBM_OK;
}

template <typename R>
int drift_run(lbm_ctx* c, R* f, const R* feq) {
    if (f == feq) return fail(c, LBM_ERR_ARG, "drift: f and feq must be distinct buffers");
    if (c->p.nl == 27) k_ref_drift<27, R><<<dim3(c->p.ny, c->p.nz), 256, 0, c->stream>>>(f, feq, c->rg);
    else k_ref_drift<19, R><<<dim3(c->p.ny, c->p.nz), 256, 0, c->stream>>>(f, feq, c->rg);
    c->launches++;
    LBM_LAUNCHED(c, "drift");
    return LBM_OK;
}

template <typename R>
int macrovars_run(lbm_ctx* c, R* rho, R* u, R* v, R* w, const R* f) {
    dim3 grd((c->p.nx + 2 + 127) / 128, c->p.ny + 2, c->p.nz + 2);
    if (c->p.nl == 27) k_ref_macrovars<27, R><<<grd, 128, 0, c->stream>>>(rho, u, v, w, f, c->rg);
    else k_ref_macrovars<19, R><<<grd, 128, 0, c->stream>>>(rho, u, v, w, f, c->rg);
    c->launches++;
    LBM_LAUNCHED(c, "macrovars");
    return LBM_OK;
}

template <typename R>
int regularization_run(lbm_ctx* c, R* f, const R* feq, const R* u, const R* v, const R* w) {
    if (c->p.nl == 27) k_ref_regularization<27, R><<<interior_rows(c), 128, 0, c->stream>>>(f, feq, u, v, w, c->rg);
    else k_ref_regularization<19, R><<<interior_rows(c), 128, 0, c->stream>>>(f, feq, u, v, w, c->rg);
    c->launches++;
    LBM_LAUNCHED(c, "regularization");
    return LBM_OK;
}

template <typename R>
int vreman_run(lbm_ctx* c, const R* f, R* tau) {
    if (c->p.ivreman != 1) return LBM_OK;   // m_vreman.F90:29-31
    const CollideParamsT<R>& cp = cp_of<R>(c);
    if (c->p.nl == 27) k_ref_vreman<27, R><<<interior_rows(c), 128, 0, c->stream>>>(f, tau, c->rg, cp);
    else k_ref_vreman<19, R><<<interior_rows(c), 128, 0, c->stream>>>(f, tau, c->rg, cp);
    c->launches++;
    LBM_LAUNCHED(c, "vreman");
    return LBM_OK;
}

// compute_fneq (sgn < 0) / compute_f (sgn > 0)
template <typename R>
int axpy_run(lbm_ctx* c, R* f, const R* feq, int sgn, const char* what) {
    const long long n = c->rg.ncell() * c->p.nl;
    k_ref_axpy<R><<<148 * 8, 256, 0, c->stream>>>(f, feq, n, sgn);
    c->launches++;
    LBM_LAUNCHED(c, what);
    return LBM_OK;
}

template <typename R>
int boundarycond_run(lbm_ctx* c, R* f1, R* f2, const R* uvel) {
    if (f1 == f2) return fail(c, LBM_ERR_ARG, "boundarycond: f1 and f2 must be distinct buffers");
    return c->p.nl == 27 ? bc_ref<27, R>(c, f1, f2, uvel) : bc_ref<19, R>(c, f1, f2, uvel);
}

template <typename R>
int forcings_apply_run(lbm_ctx* c, R* f, const R* force, const R* rho, const R* u, const R* v, const R* w) {
    if (c->p.nl == 27) k_ref_forcings_apply<27, R><<<interior_rows(c), 128, 0, c->stream>>>(f, force, rho, u, v, w, c->rg);
    else k_ref_forcings_apply<19, R><<<interior_rows(c), 128, 0, c->stream>>>(f, force, rho, u, v, w, c->rg);
    c->launches++;
    LBM_LAUNCHED(c, "forcings_apply");
    return LBM_OK;
}

template <typename R>
int solids_run(lbm_ctx* c, R* f, const int32_t* blanking) {
    if (c->p.nl == 27) k_ref_solids<27, R><<<interior_rows(c), 128, 0, c->stream>>>(f, blanking, c->rg);
    else k_ref_solids<19, R><<<interior_rows(c), 128, 0, c->stream>>>(f, blanking, c->rg);
    c->launches++;
    LBM_LAUNCHED(c, "solids");
    return LBM_OK;
}

template <typename R>
int turb_forcing_run(lbm_ctx* c, R* df, const R* rho, const R* u, const R* v, const R* w, const R* uu, const R* vv,
                     const R* ww, R ampl, int32_t it, int32_t nrturb) {
    if (nrturb <= 0) return fail(c, LBM_ERR_ARG, "inflow_turbulence_forcing: nrturb must be positive");
    if (c->p.iturb_pos < 1 || c->p.iturb_pos > c->p.nx)
        return fail(c, LBM_ERR_ARG, "inflow_turbulence_forcing: iturb_pos outside 1..nx");
    int lit = it % nrturb;   // m_inflow_turbulence_forcing.F90:45-46
    if (lit < 0) lit += nrturb;
    if (lit == 0) lit = nrturb;
    dim3 grd((c->p.ny + 127) / 128, c->p.nz);
    if (c->p.nl == 27)
        k_ref_turb_forcing<27, R><<<grd, 128, 0, c->stream>>>(df, rho, u, v, w, uu, vv, ww, ampl, lit, c->p.iturb_pos,
                                                              c->p.ibgk, c->rg);
    else
        k_ref_turb_forcing<19, R><<<grd, 128, 0, c->stream>>>(df, rho, u, v, w, uu, vv, ww, ampl, lit, c->p.iturb_pos,
                                                              c->p.ibgk, c->rg);
    c->launches++;
    LBM_LAUNCHED(c, "inflow_turbulence_forcing");
    return LBM_OK;
}

template <typename R>
int turb_apply_run(lbm_ctx* c, R* f, const R* df) {
    if (c->p.iturb_pos < 1 || c->p.iturb_pos > c->p.nx)
        return fail(c, LBM_ERR_ARG, "inflow_turbulence_apply: iturb_pos outside 1..nx");
    dim3 grd((c->p.nl * c->p.ny + 255) / 256, c->p.nz);
    k_ref_turb_apply<R><<<grd, 256, 0, c->stream>>>(f, df, c->p.iturb_pos, c->rg);
    c->launches++;
    LBM_LAUNCHED(c, "inflow_turbulence_apply");
    return LBM_OK;
}

template <typename R>
int fillghosts_run(lbm_ctx* c, R* f) {
    dim3 grd((c->p.nx + 2 + 127) / 128, c->p.ny + 2, c->p.nz + 2);
    k_ref_fillghosts<R><<<grd, 128, 0, c->stream>>>(f, c->rg);
    c->launches++;
    LBM_LAUNCHED(c, "fillghosts");
    return LBM_OK;
}

}  // namespace

// =============================================================================
extern "C" {

int lbm_abi_version(void) { return LBM_B200_ABI_VERSION; }

const char* lbm_last_error(const lbm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int lbm_create(lbm_ctx** out, const lbm_params* p) {
    if (!out || !p) return LBM_ERR_ARG;
    *out = nullptr;
    if (p->nl != 19 && p->nl != 27) return LBM_ERR_UNSUPPORTED;
    if (p->nx < 2 || p->ny < 2 || p->nz < 2) return LBM_ERR_ARG;
    if ((long long)(p->nx + 2) * (p->ny + 2) * (p->nz + 2) * p->nl >= (1LL << 40)) return LBM_ERR_ARG;
    if (p->ibgk != 2 && p->ibgk != 3) return LBM_ERR_UNSUPPORTED;
    if ((p->ihrr != 0 && p->ihrr != 1) || (p->ivreman != 0 && p->ivreman != 1)) return LBM_ERR_UNSUPPORTED;
    if (p->storage != LBM_STORE_F32 && p->storage != LBM_STORE_F16) return LBM_ERR_UNSUPPORTED;
    if (p->ibnd == 1 && (p->iturb_pos < 1 || p->iturb_pos > p->nx)) return LBM_ERR_ARG;
    lbm_ctx* c = new lbm_ctx();
    c->p = *p;
    c->rg = RefGrid{p->nx, p->ny, p->nz, p->nl};
    c->sg = SoaGrid::make(p->nx, p->ny, p->nz);
    c->cp.kinevisc = p->kinevisc;
    c->cp.cvre = 2.5f * p->smagorinsky * p->smagorinsky;
    c->cp.eps = sqrtf(1.17549435e-38f);
    c->cp.tau0 = 3.0f * p->kinevisc + 0.5f;
    c->cp.ibgk = p->ibgk;
    c->cp.ihrr = p->ihrr;
    c->cp.ivreman = p->ivreman;
    set_params_f64(c, p->kinevisc, p->smagorinsky, p->rho0, p->udir);
    c->elem = (p->storage == LBM_STORE_F16) ? 2 : 4;
    c->idx32 = (long long)p->nl * c->sg.dstride < (1LL << 31);
    setup_boundaries(c);
    int rc = LBM_OK;
    auto chk = [&](cudaError_t e, const char* w) {
        if (rc == LBM_OK && e != cudaSuccess) rc = cuda_check(c, e, w);
    };
    chk(cudaGetDevice(&c->dev), "cudaGetDevice");
    if (rc == LBM_OK) chk(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->dev), "cudaDeviceGetAttribute");
    c->stream = nullptr;
    const size_t nbuf = state_bytes_of(c);
    for (int b = 0; b < 2 && rc == LBM_OK; ++b) {
        chk(cudaMalloc(&c->own[b], nbuf), "cudaMalloc(state)");
        if (rc == LBM_OK) chk(cudaMemset(c->own[b], 0, nbuf), "cudaMemset(state)");
        c->buf[b] = c->own[b];
    }
    const size_t g = (size_t)c->rg.ncell();
    chk(cudaMalloc(&c->d_macro, 4 * g * sizeof(float)), "cudaMalloc(macro)");
    chk(cudaMalloc(&c->d_uvel, (size_t)p->nz * sizeof(float)), "cudaMalloc(uvel)");
    chk(cudaMalloc(&c->d_edge, (size_t)2 * p->nl * p->ny * p->nz * c->elem), "cudaMalloc(edge)");
    for (int b = 0; b < 2 && c->fold; ++b)
        chk(cudaMalloc(&c->d_xg[b], (size_t)2 * p->nl * p->ny * p->nz * c->elem), "cudaMalloc(x-ghost)");
    chk(cudaMalloc(&c->d_abl, (size_t)p->nz * sizeof(float)), "cudaMalloc(ablvisc)");
    chk(cudaMalloc(&c->d_it, 2 * sizeof(int)), "cudaMalloc(step)");
    chk(cudaMalloc(&c->d_status, sizeof(int)), "cudaMalloc(status)");
    chk(cudaMalloc(&c->d_partial, (size_t)LBM_SUM_BLOCKS * 4 * sizeof(double)), "cudaMalloc(partial)");
    chk(cudaMalloc(&c->d_sum, 4 * sizeof(double)), "cudaMalloc(sum)");
    if (rc == LBM_OK) {
        chk(cudaMemset(c->d_uvel, 0, (size_t)p->nz * sizeof(float)), "cudaMemset");
        chk(cudaMemset(c->d_abl, 0, (size_t)p->nz * sizeof(float)), "cudaMemset");
        chk(cudaMemset(c->d_it, 0, 2 * sizeof(int)), "cudaMemset");
        chk(cudaMemset(c->d_status, 0, sizeof(int)), "cudaMemset");
        chk(cudaDeviceSynchronize(), "create");
    }
    if (rc != LBM_OK) {
        lbm_destroy(c);
        return rc;
    }
    *out = c;
    return LBM_OK;
}

int lbm_destroy(lbm_ctx* c) {
    if (!c) return LBM_ERR_ARG;
    cudaStreamSynchronize(c->stream);
    for (cudaEvent_t e : c->ev) cudaEventDestroy(e);
    for (int b = 0; b < 2; ++b) cudaFree(c->own[b]);
    cudaFree(c->d_macro);
    cudaFree(c->d_solid);
    cudaFree(c->d_turb);
    cudaFree(c->d_uvel);
    cudaFree(c->d_edge);
    for (int b = 0; b < 2; ++b) cudaFree(c->d_xg[b]);
    cudaFree(c->d_abl);
    cudaFree(c->d_adj_terms);
    cudaFree(c->d_it);
    cudaFree(c->d_status);
    cudaFree(c->d_partial);
    cudaFree(c->d_sum);
    delete c;
    return LBM_OK;
}

int lbm_set_stream(lbm_ctx* c, void* stream) {
    if (!c) return LBM_ERR_ARG;
    c->stream = (cudaStream_t)stream;
    return LBM_OK;
}

int lbm_synchronize(lbm_ctx* c) {
    if (!c) return LBM_ERR_ARG;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "synchronize");
}

// ---- per-call entry points (FP32; the _f64 forms take the DP build's arrays) ----
// Each pair checks its pointers and runs the same kernels in its own type.

int lbm_fequil3(lbm_ctx* c, float* feq, const float* rho, const float* u, const float* v, const float* w) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, feq); NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w);
    return fequil3_run(c, feq, rho, u, v, w);
}
int lbm_fequil3_f64(lbm_ctx* c, double* feq, const double* rho, const double* u, const double* v, const double* w) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, feq); NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w);
    return fequil3_run(c, feq, rho, u, v, w);
}

int lbm_postcoll(lbm_ctx* c, float* f, float* tau, const float* rho, const float* u, const float* v, const float* w,
                 const float* ablvisc) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, tau); NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w);
    return postcoll_run(c, f, tau, rho, u, v, w, ablvisc);
}
int lbm_postcoll_f64(lbm_ctx* c, double* f, double* tau, const double* rho, const double* u, const double* v,
                     const double* w, const double* ablvisc) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, tau); NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w);
    return postcoll_run(c, f, tau, rho, u, v, w, ablvisc);
}

int lbm_drift(lbm_ctx* c, float* f, const float* feq) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, feq);
    return drift_run(c, f, feq);
}
int lbm_drift_f64(lbm_ctx* c, double* f, const double* feq) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, feq);
    return drift_run(c, f, feq);
}

int lbm_macrovars(lbm_ctx* c, float* rho, float* u, float* v, float* w, const float* f) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w); NEED(c, f);
    return macrovars_run(c, rho, u, v, w, f);
}
int lbm_macrovars_f64(lbm_ctx* c, double* rho, double* u, double* v, double* w, const double* f) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w); NEED(c, f);
    return macrovars_run(c, rho, u, v, w, f);
}

int lbm_regularization(lbm_ctx* c, float* f, const float* feq, const float* u, const float* v, const float* w) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, feq); NEED(c, u); NEED(c, v); NEED(c, w);
    return regularization_run(c, f, feq, u, v, w);
}
int lbm_regularization_f64(lbm_ctx* c, double* f, const double* feq, const double* u, const double* v,
                           const double* w) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, feq); NEED(c, u); NEED(c, v); NEED(c, w);
    return regularization_run(c, f, feq, u, v, w);
}

int lbm_vreman(lbm_ctx* c, const float* f, float* tau) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, tau);
    return vreman_run(c, f, tau);
}
int lbm_vreman_f64(lbm_ctx* c, const double* f, double* tau) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, tau);
    return vreman_run(c, f, tau);
}

int lbm_compute_fneq(lbm_ctx* c, float* f, const float* feq) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, feq);
    return axpy_run(c, f, feq, -1, "compute_fneq");
}
int lbm_compute_fneq_f64(lbm_ctx* c, double* f, const double* feq) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, feq);
    return axpy_run(c, f, feq, -1, "compute_fneq");
}
int lbm_compute_f(lbm_ctx* c, float* f, const float* feq) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, feq);
    return axpy_run(c, f, feq, 1, "compute_f");
}
int lbm_compute_f_f64(lbm_ctx* c, double* f, const double* feq) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, feq);
    return axpy_run(c, f, feq, 1, "compute_f");
}

int lbm_boundarycond(lbm_ctx* c, float* f1, float* f2, const float* uvel) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f1); NEED(c, f2);
    if (c->p.ibnd == 1) NEED(c, uvel);
    return boundarycond_run(c, f1, f2, uvel);
}
int lbm_boundarycond_f64(lbm_ctx* c, double* f1, double* f2, const double* uvel) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f1); NEED(c, f2);
    if (c->p.ibnd == 1) NEED(c, uvel);
    return boundarycond_run(c, f1, f2, uvel);
}

int lbm_forcings_apply(lbm_ctx* c, float* f, const float* external_forcing, const float* rho, const float* u,
                       const float* v, const float* w) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, external_forcing); NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w);
    return forcings_apply_run(c, f, external_forcing, rho, u, v, w);
}
int lbm_forcings_apply_f64(lbm_ctx* c, double* f, const double* external_forcing, const double* rho,
                           const double* u, const double* v, const double* w) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, external_forcing); NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w);
    return forcings_apply_run(c, f, external_forcing, rho, u, v, w);
}

int lbm_set_forcing(lbm_ctx* c, const float* external_forcing) {
    if (!c) return LBM_ERR_ARG;
    c->force = external_forcing;
    return LBM_OK;
}

int lbm_solids(lbm_ctx* c, float* f, const int32_t* blanking) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, blanking);
    return solids_run(c, f, blanking);
}
int lbm_solids_f64(lbm_ctx* c, double* f, const int32_t* blanking) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, blanking);
    return solids_run(c, f, blanking);
}

int lbm_inflow_turbulence_forcing(lbm_ctx* c, float* df, const float* rho, const float* u, const float* v,
                                  const float* w, const float* uu, const float* vv, const float* ww, float ampl,
                                  int32_t it, int32_t nrturb) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, df); NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w); NEED(c, uu); NEED(c, vv); NEED(c, ww);
    return turb_forcing_run(c, df, rho, u, v, w, uu, vv, ww, ampl, it, nrturb);
}
int lbm_inflow_turbulence_forcing_f64(lbm_ctx* c, double* df, const double* rho, const double* u, const double* v,
                                      const double* w, const double* uu, const double* vv, const double* ww,
                                      double ampl, int32_t it, int32_t nrturb) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, df); NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w); NEED(c, uu); NEED(c, vv); NEED(c, ww);
    return turb_forcing_run(c, df, rho, u, v, w, uu, vv, ww, ampl, it, nrturb);
}

int lbm_inflow_turbulence_apply(lbm_ctx* c, float* f, const float* df) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, df);
    return turb_apply_run(c, f, df);
}
int lbm_inflow_turbulence_apply_f64(lbm_ctx* c, double* f, const double* df) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, df);
    return turb_apply_run(c, f, df);
}

int lbm_fillghosts(lbm_ctx* c, float* f) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f);
    return fillghosts_run(c, f);
}
int lbm_fillghosts_f64(lbm_ctx* c, double* f) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f);
    return fillghosts_run(c, f);
}

int lbm_set_params_f64(lbm_ctx* c, double kinevisc, double smagorinsky, double rho0, double udir) {
    if (!c) return LBM_ERR_ARG;
    set_params_f64(c, kinevisc, smagorinsky, rho0, udir);
    return LBM_OK;
}

// ---- fused state API -----------------------------------------------------------

int lbm_state_import(lbm_ctx* c, const float* f1, const float* f2, const float* rho, const float* u, const float* v,
                     const float* w, int32_t it) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f1); NEED(c, f2); NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w);
    c->buf[0] = c->own[0];
    c->buf[1] = c->own[1];
    DISPATCH_QS(c, launch_import, c, f1, 0);
    DISPATCH_QS(c, launch_import, c, f2, 1);
    const size_t g = (size_t)c->rg.ncell() * sizeof(float);
    const float* src[4] = {rho, u, v, w};
    for (int q = 0; q < 4; ++q)
        LBM_TRY(cuda_check(c, cudaMemcpyAsync((char*)c->d_macro + q * g, src[q], g, cudaMemcpyDeviceToDevice, c->stream),
                           "import macro"));
    const int nxt = it + 1;
    LBM_TRY(cuda_check(c, cudaMemcpyAsync(c->d_it, &nxt, sizeof(int), cudaMemcpyHostToDevice, c->stream), "import step"));
    LBM_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "import"));
    LBM_LAUNCHED(c, "import");
    c->cur = 0;
    c->it = it;
    c->state = ST_PRE;
    return LBM_OK;
}

int lbm_state_export(lbm_ctx* c, float* f1, float* f2) {
    if (!c) return LBM_ERR_ARG;
    if (c->state == ST_NONE) return fail(c, LBM_ERR_STATE, "state_export: no state imported");
    NEED(c, f1); NEED(c, f2);
    const bool post = (c->state == ST_POST);
    if (post) {
        DISPATCH_QS(c, launch_export, c, f1, c->cur, true);
        DISPATCH_QS(c, launch_export, c, f2, c->cur, false);
    } else {
        DISPATCH_QS(c, launch_export, c, f1, c->cur, false);
        DISPATCH_QS(c, launch_export, c, f2, 1 - c->cur, false);
    }
    LBM_LAUNCHED(c, "export");
    return LBM_OK;
}

int lbm_get_macro(lbm_ctx* c, float* rho, float* u, float* v, float* w) {
    if (!c) return LBM_ERR_ARG;
    if (c->state == ST_NONE) return fail(c, LBM_ERR_STATE, "get_macro: no state imported");
    NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w);
    if (c->state == ST_PRE) {
        const size_t g = (size_t)c->rg.ncell() * sizeof(float);
        float* dst[4] = {rho, u, v, w};
        for (int q = 0; q < 4; ++q)
            LBM_TRY(cuda_check(c, cudaMemcpyAsync(dst[q], (char*)c->d_macro + q * g, g, cudaMemcpyDeviceToDevice,
                                                  c->stream), "get_macro"));
        return LBM_OK;
    }
    DISPATCH_QS(c, launch_macro, c, rho, u, v, w);
    LBM_LAUNCHED(c, "get_macro");
    return LBM_OK;
}

__global__ void k_mask_from_logical(uint8_t* m, const int32_t* blank, RefGrid g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
    if (i > g.nx) return;
    m[((long long)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1)] = blank[g.cell(i, j, k)] != 0;
}

int lbm_set_solids(lbm_ctx* c, const int32_t* blanking) {
    if (!c) return LBM_ERR_ARG;
    if (!blanking) {
        LBM_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "set_solids"));
        cudaFree(c->d_solid);
        c->d_solid = nullptr;
        return LBM_OK;
    }
    if (!c->d_solid)
        LBM_TRY(cuda_check(c, cudaMalloc(&c->d_solid, (size_t)c->p.nx * c->p.ny * c->p.nz), "cudaMalloc(solids)"));
    dim3 grd((c->p.nx + 127) / 128, c->p.ny, c->p.nz);
    k_mask_from_logical<<<grd, 128, 0, c->stream>>>(c->d_solid, blanking, c->rg);
    c->launches++;
    LBM_LAUNCHED(c, "set_solids");
    return LBM_OK;
}

int lbm_set_turbulence(lbm_ctx* c, const float* uu, const float* vv, const float* ww, int32_t nrturb, float ampl) {
    if (!c) return LBM_ERR_ARG;
    if (!uu) {
        LBM_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "set_turbulence"));
        cudaFree(c->d_turb);
        c->d_turb = nullptr;
        c->nrturb = 0;
        return LBM_OK;
    }
    NEED(c, vv); NEED(c, ww);
    if (nrturb <= 0) return fail(c, LBM_ERR_ARG, "set_turbulence: nrturb must be positive");
    if (c->p.iturb_pos < 1 || c->p.iturb_pos > c->p.nx)
        return fail(c, LBM_ERR_ARG, "set_turbulence: iturb_pos outside 1..nx");
    const size_t n = (size_t)c->p.ny * c->p.nz * (nrturb + 1);
    LBM_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "set_turbulence"));
    cudaFree(c->d_turb);
    c->d_turb = nullptr;
    LBM_TRY(cuda_check(c, cudaMalloc(&c->d_turb, 3 * n * sizeof(float)), "cudaMalloc(turbulence)"));
    const float* src[3] = {uu, vv, ww};
    for (int q = 0; q < 3; ++q)
        LBM_TRY(cuda_check(c, cudaMemcpyAsync(c->d_turb + q * n, src[q], n * sizeof(float), cudaMemcpyDeviceToDevice,
                                              c->stream), "set_turbulence"));
    c->nrturb = nrturb;
    c->ampl = ampl;
    return LBM_OK;
}

int lbm_set_inflow(lbm_ctx* c, const float* uvel) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, uvel);
    return cuda_check(c, cudaMemcpyAsync(c->d_uvel, uvel, (size_t)c->p.nz * sizeof(float), cudaMemcpyDeviceToDevice,
                                         c->stream), "set_inflow");
}

int lbm_step(lbm_ctx* c, int32_t nsteps) {
    if (!c) return LBM_ERR_ARG;
    if (c->state == ST_NONE) return fail(c, LBM_ERR_STATE, "step: no state imported");
    if (nsteps < 0) return fail(c, LBM_ERR_ARG, "step: nsteps < 0");
    for (int s = 0; s < nsteps; ++s) {
        own_dst(c);
        LBM_LAUNCHED(c, "step: ghost shell");
        LBM_TRY(step_dispatch(c));
    }
    return LBM_OK;
}

int lbm_step_to(lbm_ctx* c, void* dst) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, dst);
    if (c->state == ST_NONE) return fail(c, LBM_ERR_STATE, "step_to: no state imported");
    if (reinterpret_cast<uintptr_t>(dst) % 256 != 0) return fail(c, LBM_ERR_ARG, "step_to: dst not 256-byte aligned");
    if (dst == c->buf[c->cur] || dst == c->own[0] || dst == c->own[1])
        return fail(c, LBM_ERR_ARG, "step_to: dst is one of the context's buffers");
    if (c->state == ST_PRE) {
        // the first step after an import collides in place: step, then copy
        own_dst(c);
        LBM_TRY(step_dispatch(c));
        return lbm_state_copy(c, dst);
    }
    take_dst(c, dst);
    LBM_LAUNCHED(c, "step_to: ghost shell");
    return step_dispatch(c);
}

// ---- snapshots: a stepped state kept in device memory and resumed later -------
// Layout: the current buffer (as lbm_state_copy), the ghost shell of the other
// buffer (packed, k_pack_ghosts), the x-ghost columns of both buffers (folded
// configuration) and a header.  Each part starts on a 256-byte boundary.
struct SnapLayout {
    size_t buf, shell, xg, head, total;
};
struct SnapHead {
    int32_t magic, it, nx, ny, nz, nl, storage, fold;
};
static const int32_t kSnapMagic = 0x4c424d53;   // "LBMS"

static SnapLayout snap_layout(const lbm_ctx* c) {
    auto up = [](size_t n) { return (n + 255) / 256 * 256; };
    SnapLayout L;
    L.buf = up(state_bytes_of(c));
    L.shell = up((size_t)c->p.nl * ghost_cells(c->sg) * c->elem);
    L.xg = c->fold ? up((size_t)2 * c->p.nl * c->p.ny * c->p.nz * c->elem) : 0;
    L.head = 256;
    L.total = L.buf + L.shell + 2 * L.xg + L.head;
    return L;
}

static void pack_ghosts(lbm_ctx* c, void* packed, void* buf, bool unpack) {
    const long long n = ghost_cells(c->sg);
    const dim3 grd((unsigned)((n + 127) / 128), (unsigned)c->p.nl);
    if (c->elem == 2) {
        if (unpack) k_pack_ghosts<uint16_t, true><<<grd, 128, 0, c->stream>>>((uint16_t*)packed, (uint16_t*)buf, c->sg, n);
        else k_pack_ghosts<uint16_t, false><<<grd, 128, 0, c->stream>>>((uint16_t*)packed, (uint16_t*)buf, c->sg, n);
    } else {
        if (unpack) k_pack_ghosts<uint32_t, true><<<grd, 128, 0, c->stream>>>((uint32_t*)packed, (uint32_t*)buf, c->sg, n);
        else k_pack_ghosts<uint32_t, false><<<grd, 128, 0, c->stream>>>((uint32_t*)packed, (uint32_t*)buf, c->sg, n);
    }
    c->launches++;
}

int lbm_state_snapshot_bytes(lbm_ctx* c, int64_t* bytes) {
    if (!c || !bytes) return LBM_ERR_ARG;
    *bytes = (int64_t)snap_layout(c).total;
    return LBM_OK;
}

int lbm_state_snapshot(lbm_ctx* c, void* dst) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, dst);
    if (c->state != ST_POST)
        return fail(c, LBM_ERR_STATE, "state_snapshot: no stepped state (after an import, keep its f1, f2 instead)");
    if (reinterpret_cast<uintptr_t>(dst) % 256 != 0) return fail(c, LBM_ERR_ARG, "state_snapshot: dst not 256-byte aligned");
    const SnapLayout L = snap_layout(c);
    char* d = static_cast<char*>(dst);
    const size_t nbuf = state_bytes_of(c);
    LBM_TRY(cuda_check(c, cudaMemcpyAsync(d, c->buf[c->cur], nbuf, cudaMemcpyDeviceToDevice, c->stream), "snapshot"));
    pack_ghosts(c, d + L.buf, c->buf[1 - c->cur], false);
    if (c->fold) {
        const size_t nxg = (size_t)2 * c->p.nl * c->p.ny * c->p.nz * c->elem;
        LBM_TRY(cuda_check(c, cudaMemcpyAsync(d + L.buf + L.shell, c->d_xg[c->cur], nxg, cudaMemcpyDeviceToDevice,
                                              c->stream), "snapshot"));
        LBM_TRY(cuda_check(c, cudaMemcpyAsync(d + L.buf + L.shell + L.xg, c->d_xg[1 - c->cur], nxg,
                                              cudaMemcpyDeviceToDevice, c->stream), "snapshot"));
    }
    const SnapHead h{kSnapMagic, c->it, c->p.nx, c->p.ny, c->p.nz, c->p.nl, c->p.storage, c->fold ? 1 : 0};
    LBM_TRY(cuda_check(c, cudaMemcpyAsync(d + L.buf + L.shell + 2 * L.xg, &h, sizeof(h), cudaMemcpyHostToDevice,
                                          c->stream), "snapshot"));
    LBM_LAUNCHED(c, "snapshot");
    return LBM_OK;
}

int lbm_state_restore(lbm_ctx* c, const void* src) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, src);
    if (reinterpret_cast<uintptr_t>(src) % 256 != 0) return fail(c, LBM_ERR_ARG, "state_restore: src not 256-byte aligned");
    const SnapLayout L = snap_layout(c);
    const char* s = static_cast<const char*>(src);
    SnapHead h;
    LBM_TRY(cuda_check(c, cudaMemcpyAsync(&h, s + L.buf + L.shell + 2 * L.xg, sizeof(h), cudaMemcpyDeviceToHost,
                                          c->stream), "restore"));
    LBM_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "restore"));
    if (h.magic != kSnapMagic || h.nx != c->p.nx || h.ny != c->p.ny || h.nz != c->p.nz || h.nl != c->p.nl ||
        h.storage != c->p.storage || h.fold != (c->fold ? 1 : 0))
        return fail(c, LBM_ERR_ARG, "state_restore: not a snapshot of a context with these parameters");
    c->buf[0] = c->own[0];
    c->buf[1] = c->own[1];
    const size_t nbuf = state_bytes_of(c);
    LBM_TRY(cuda_check(c, cudaMemcpyAsync(c->buf[0], s, nbuf, cudaMemcpyDeviceToDevice, c->stream), "restore"));
    pack_ghosts(c, const_cast<char*>(s) + L.buf, c->buf[1], true);
    if (c->fold) {
        const size_t nxg = (size_t)2 * c->p.nl * c->p.ny * c->p.nz * c->elem;
        LBM_TRY(cuda_check(c, cudaMemcpyAsync(c->d_xg[0], s + L.buf + L.shell, nxg, cudaMemcpyDeviceToDevice, c->stream),
                           "restore"));
        LBM_TRY(cuda_check(c, cudaMemcpyAsync(c->d_xg[1], s + L.buf + L.shell + L.xg, nxg, cudaMemcpyDeviceToDevice,
                                              c->stream), "restore"));
    }
    const int nxt = h.it + 1;
    LBM_TRY(cuda_check(c, cudaMemcpyAsync(c->d_it, &nxt, sizeof(int), cudaMemcpyHostToDevice, c->stream), "restore"));
    LBM_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "restore"));
    LBM_LAUNCHED(c, "restore");
    c->cur = 0;
    c->it = h.it;
    c->state = ST_POST;
    return LBM_OK;
}

// ---- j-slab decomposition (m_mpi_halo_exchange_j.F90:3-121, m_mpi_pack_jplane.F90,
// m_mpi_unpack_jplane.F90) ---------------------------------------------------------
int lbm_set_halo_j(lbm_ctx* c, int32_t on) {
    if (!c) return LBM_ERR_ARG;
    if (c->state != ST_NONE) return fail(c, LBM_ERR_STATE, "set_halo_j: call it before the first import");
    c->halo_j = (on != 0);
    return LBM_OK;
}

int lbm_halo_plane_bytes(lbm_ctx* c, int64_t* bytes) {
    if (!c || !bytes) return LBM_ERR_ARG;
    *bytes = (int64_t)c->p.nl * (c->p.nx + 2) * (c->p.nz + 2) * (int64_t)c->elem;
    return LBM_OK;
}

static int halo_plane(lbm_ctx* c, void* buf, int j, bool unpack) {
    const long long n = (long long)c->p.nl * (c->p.nz + 2) * (c->p.nx + 2);
    const unsigned grd = (unsigned)((n + 255) / 256);
    const int Q = c->p.nl;
    void* f = c->buf[c->cur];
    // folded configuration after a step: the x ghosts of every direction are in the compact array
    const void* xg = (c->fold && c->state == ST_POST) ? c->d_xg[c->cur] : nullptr;
    if (c->elem == 2) {
        if (unpack) k_halo_plane<uint16_t, true><<<grd, 256, 0, c->stream>>>((uint16_t*)buf, (uint16_t*)f, c->sg, j, Q, nullptr);
        else k_halo_plane<uint16_t, false><<<grd, 256, 0, c->stream>>>((uint16_t*)buf, (uint16_t*)f, c->sg, j, Q, (const uint16_t*)xg);
    } else {
        if (unpack) k_halo_plane<uint32_t, true><<<grd, 256, 0, c->stream>>>((uint32_t*)buf, (uint32_t*)f, c->sg, j, Q, nullptr);
        else k_halo_plane<uint32_t, false><<<grd, 256, 0, c->stream>>>((uint32_t*)buf, (uint32_t*)f, c->sg, j, Q, (const uint32_t*)xg);
    }
    c->launches++;
    return LBM_OK;
}

int lbm_halo_pack_j(lbm_ctx* c, void* to_south, void* to_north) {
    if (!c) return LBM_ERR_ARG;
    if (!c->halo_j) return fail(c, LBM_ERR_STATE, "halo_pack_j: lbm_set_halo_j(ctx, 1) was not called");
    if (c->state == ST_NONE) return fail(c, LBM_ERR_STATE, "halo_pack_j: no state imported");
    if (to_south) halo_plane(c, to_south, 1, false);
    if (to_north) halo_plane(c, to_north, c->p.ny, false);
    LBM_LAUNCHED(c, "halo pack");
    return LBM_OK;
}

int lbm_halo_unpack_j(lbm_ctx* c, const void* from_south, const void* from_north) {
    if (!c) return LBM_ERR_ARG;
    if (!c->halo_j) return fail(c, LBM_ERR_STATE, "halo_unpack_j: lbm_set_halo_j(ctx, 1) was not called");
    if (c->state == ST_NONE) return fail(c, LBM_ERR_STATE, "halo_unpack_j: no state imported");
    if (from_south) halo_plane(c, const_cast<void*>(from_south), 0, true);
    if (from_north) halo_plane(c, const_cast<void*>(from_north), c->p.ny + 1, true);
    LBM_LAUNCHED(c, "halo unpack");
    return LBM_OK;
}

int lbm_step_host(lbm_ctx* c, int32_t nsteps, const float* uvel_host, int32_t* status_host) {
    if (!c) return LBM_ERR_ARG;
    if (c->state == ST_NONE) return fail(c, LBM_ERR_STATE, "step_host: no state imported");
    if (nsteps < 0) return fail(c, LBM_ERR_ARG, "step_host: nsteps < 0");
    for (int s = 0; s < nsteps; ++s) {
        if (uvel_host)
            LBM_TRY(cuda_check(c, cudaMemcpyAsync(c->d_uvel, uvel_host, (size_t)c->p.nz * sizeof(float),
                                                  cudaMemcpyHostToDevice, c->stream), "step_host uvel"));
        own_dst(c);
        LBM_TRY(step_dispatch(c));
    }
    if (status_host) {
        LBM_TRY(cuda_check(c, cudaMemcpyAsync(status_host, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                           "step_host status"));
        LBM_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "step_host"));
    }
    return LBM_OK;
}

int lbm_get_step(lbm_ctx* c, int32_t* it) {
    if (!c || !it) return LBM_ERR_ARG;
    *it = c->it;
    return LBM_OK;
}

int lbm_mass_momentum(lbm_ctx* c, const float* f, double* out) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f); NEED(c, out);
    if (c->p.nl == 27) k_sum_ref<27><<<LBM_SUM_BLOCKS, 256, 0, c->stream>>>(f, c->rg, c->d_partial);
    else k_sum_ref<19><<<LBM_SUM_BLOCKS, 256, 0, c->stream>>>(f, c->rg, c->d_partial);
    c->launches++;
    k_sum_final<<<1, 256, 0, c->stream>>>(c->d_partial, LBM_SUM_BLOCKS, out);
    c->launches++;
    LBM_LAUNCHED(c, "mass_momentum");
    return LBM_OK;
}

int lbm_conservation(lbm_ctx* c, double* out_host) {
    if (!c || !out_host) return LBM_ERR_ARG;
    if (c->state == ST_NONE) return fail(c, LBM_ERR_STATE, "conservation: no state imported");
    if (c->state == ST_POST) {
        DISPATCH_QS(c, launch_sum_state, c);
    } else {
        DISPATCH_QS(c, launch_sum_pre, c);
    }
    k_sum_final<<<1, 256, 0, c->stream>>>(c->d_partial, LBM_SUM_BLOCKS, c->d_sum);
    c->launches++;
    LBM_LAUNCHED(c, "conservation");
    LBM_TRY(cuda_check(c, cudaMemcpyAsync(out_host, c->d_sum, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                       "conservation"));
    return cuda_check(c, cudaStreamSynchronize(c->stream), "conservation");
}

// Device address of g_noalloc_partial on the current device, looked up once per
// device (host code may not use the symbol itself as an address).  The cached
// address belongs to the device's current context: a caller that resets the
// device (cudaDeviceReset) cannot use this entry point afterwards.
static int noalloc_scratch(double** out) {
    static std::mutex mu;
    static double* addr[128] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return LBM_ERR_CUDA;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_partial) != cudaSuccess || !p) return LBM_ERR_CUDA;
        addr[dev] = (double*)p;
    }
    *out = addr[dev];
    return LBM_OK;
}

int lbm_mass_momentum_noalloc(const float* f, int32_t nx, int32_t ny, int32_t nz, int32_t nl, double* out,
                              void* stream) {
    if (!f || !out) return LBM_ERR_ARG;
    if (nl != 19 && nl != 27) return LBM_ERR_UNSUPPORTED;
    if (nx < 1 || ny < 1 || nz < 1) return LBM_ERR_ARG;
    const long long cells = (long long)nx * ny * nz;
    const long long nblocks = (cells + LBM_NOALLOC_CHUNK - 1) / LBM_NOALLOC_CHUNK;
    if (nblocks > LBM_NOALLOC_BLOCKS) return LBM_ERR_ARG;     // more than 134,217,728 interior cells
    double* scratch = nullptr;
    const int rc = noalloc_scratch(&scratch);
    if (rc != LBM_OK) return rc;
    RefGrid g{nx, ny, nz, nl};
    cudaStream_t s = (cudaStream_t)stream;
    // cudaLaunchKernel returns this launch's own error, not an error left pending by
    // the caller's earlier work (a sticky error of a broken context is reported, as
    // by every CUDA call)
    int nb = (int)nblocks;
    void* sum_args[] = {(void*)&f, (void*)&g, (void*)&scratch};
    const void* ksum = (nl == 27) ? (const void*)k_sum_ref<27> : (const void*)k_sum_ref<19>;
    if (cudaLaunchKernel(ksum, dim3((unsigned)nb), dim3(256), sum_args, 0, s) != cudaSuccess) return LBM_ERR_CUDA;
    void* fin_args[] = {(void*)&scratch, (void*)&nb, (void*)&out};
    if (cudaLaunchKernel((const void*)k_sum_final, dim3(1), dim3(256), fin_args, 0, s) != cudaSuccess)
        return LBM_ERR_CUDA;
    return LBM_OK;
}

int lbm_set_kernel(lbm_ctx* c, int32_t which) {
    if (!c) return LBM_ERR_ARG;
    if (which != LBM_KERNEL_PULL && which != LBM_KERNEL_PAIR)
        return fail(c, LBM_ERR_ARG, "set_kernel: unknown kernel");
    c->kernel = which;
    return LBM_OK;
}

int lbm_launch_count(lbm_ctx* c, int64_t* n) {
    if (!c || !n) return LBM_ERR_ARG;
    *n = c->launches;
    return LBM_OK;
}

int lbm_profile(lbm_ctx* c, int32_t enable) {
    if (!c) return LBM_ERR_ARG;
    if (enable && c->ev.empty()) {
        c->ev.resize(2 * 1024);
        for (auto& e : c->ev) LBM_TRY(cuda_check(c, cudaEventCreate(&e), "cudaEventCreate"));
    }
    LBM_TRY(prof_drain(c));
    c->profiling = enable != 0;
    c->prof_ms = 0.0;
    c->prof_bc_ms = 0.0;
    c->prof_launches = 0;
    return LBM_OK;
}

int lbm_profile_read(lbm_ctx* c, double* step_kernel_ms, int64_t* step_kernel_launches) {
    if (!c || !step_kernel_ms || !step_kernel_launches) return LBM_ERR_ARG;
    LBM_TRY(prof_drain(c));
    *step_kernel_ms = c->prof_ms;
    *step_kernel_launches = c->prof_launches;
    return LBM_OK;
}

int lbm_profile_read_boundary(lbm_ctx* c, double* boundary_ms, int64_t* steps) {
    if (!c || !boundary_ms || !steps) return LBM_ERR_ARG;
    LBM_TRY(prof_drain(c));
    *boundary_ms = c->prof_bc_ms;
    *steps = c->prof_launches;
    return LBM_OK;
}

int lbm_status(lbm_ctx* c, int32_t* flags) {
    if (!c || !flags) return LBM_ERR_ARG;
    LBM_TRY(cuda_check(c, cudaMemcpyAsync(flags, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "status"));
    LBM_TRY(cuda_check(c, cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream), "status"));
    LBM_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "status"));
    return LBM_OK;
}

}  // extern "C"

#include "ensemble_host.cuh"
#include "adjoint_host.cuh"
#include "turbulence_host.cuh"
