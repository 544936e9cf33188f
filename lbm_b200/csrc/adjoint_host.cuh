// adjoint_host.cuh -- C ABI of the adjoint kernels (declarations in
// include/lbm_b200.h).  Included at the end of api.cu, whose lbm_ctx and
// boundary tables it uses.

#include "adjoint.cuh"
#include "adjoint_state.cuh"

namespace {

// boundarycond in reverse: the launches of run_bc in the opposite order, each
// with the adjoint accessor (a copy becomes an accumulation into its source).
// wrap: the accessors read periodic j ghost rows as rows ny and 1, so the j copies
// are identities (left out) and the other copies skip those rows.
template <int Q, typename AdjA>
int run_bc_adj(lbm_ctx* c, AdjA a1, AdjA a2, float* uvelh, bool wrap = false) {
    const int nx = c->p.nx, ny = c->p.ny, nz = c->p.nz, nl = c->p.nl;
    cudaStream_t s = c->stream;
    auto periodic = [&](int axis) {
        dim3 grd;
        if (axis == 0) grd = dim3((ny + 2 + 127) / 128, nz + 2, nl);
        else if (axis == 1) grd = dim3((nx + 2 + 127) / 128, nz + 2, nl);
        else grd = dim3((nx + 2 + 127) / 128, ny + 2, nl);
        k_periodic_adj<AdjA><<<grd, 128, 0, s>>>(a1, axis, nl, wrap ? 1 : 0);
        c->launches++;
    };
    const int codes[3] = {c->p.ibnd, c->p.jbnd, c->p.kbnd};
    for (int a = 2; a >= 0; --a)
        if (codes[a] == 0 && !(wrap && a == 1)) periodic(a);
    if (c->p.ibnd == 1) {
        k_inflow_adj<Q, AdjA><<<dim3((ny + 31) / 32, nz), 32, 0, s>>>(a1, uvelh, c->p.rho0, c->cosd, c->sind);
        c->launches++;
    }
    if (c->corners_on) {
        k_corners<AdjA><<<1, 32, 0, s>>>(a1, a2, c->corners);
        c->launches++;
    }
    for (int e = 2; e >= 0; --e) {
        if (!c->edges_on[e]) continue;
        const EdgeSet& es = c->edges[e];
        k_edges<AdjA><<<dim3((es.nfree + 127) / 128, 4), 128, 0, s>>>(a1, a2, es);
        c->launches++;
    }
    for (int a = 2; a >= 0; --a) {
        if (!c->face_on[a]) continue;
        const int na = (a == 0) ? ny : nx;
        const int nb = (a == 2) ? ny : nz;
        k_closed_adj<AdjA><<<dim3((na + 127) / 128, nb, 2), 128, 0, s>>>(a1, a2, a, c->face[a][0], c->face[a][1]);
        c->launches++;
    }
    for (int a = 2; a >= 0; --a)
        if (codes[a] == 0 && !(wrap && a == 1)) periodic(a);
    LBM_LAUNCHED(c, "boundarycond adjoint");
    return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_postcoll_adj(lbm_ctx* c, float* fhat, const float* f, const float* tau, const float* rho, const float* u,
                     const float* v, const float* w, const float* ablvisc, float* rhohat, float* uhat, float* vhat,
                     float* what, const int32_t* blanking) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, fhat); NEED(c, f); NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w);
    NEED(c, rhohat); NEED(c, uhat); NEED(c, vhat); NEED(c, what);
    if (!c->p.ivreman) NEED(c, tau);
    if (c->p.ihrr != 1)
        return fail(c, LBM_ERR_UNSUPPORTED, "postcoll_adj: the adjoint covers the regularized collision (ihrr = 1)");
    dim3 grd((c->p.nx + 127) / 128, c->p.ny, c->p.nz);
    // with Vreman the forward computes tau itself; any array stands in for the unused input
    const float* t = tau ? tau : rho;
    if (c->p.nl == 27)
        k_ref_postcoll_adj<27><<<grd, 128, 0, c->stream>>>(fhat, f, rho, u, v, w, t, ablvisc, rhohat, uhat, vhat, what,
                                                           blanking, c->rg, c->cp);
    else
        k_ref_postcoll_adj<19><<<grd, 128, 0, c->stream>>>(fhat, f, rho, u, v, w, t, ablvisc, rhohat, uhat, vhat, what,
                                                           blanking, c->rg, c->cp);
    c->launches++;
    LBM_LAUNCHED(c, "postcoll adjoint");
    return LBM_OK;
}

int lbm_macrovars_adj(lbm_ctx* c, float* fhat, const float* rhohat, const float* uhat, const float* vhat,
                      const float* what, const float* f) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, fhat); NEED(c, rhohat); NEED(c, uhat); NEED(c, vhat); NEED(c, what); NEED(c, f);
    dim3 grd((c->p.nx + 2 + 127) / 128, c->p.ny + 2, c->p.nz + 2);
    if (c->p.nl == 27) k_ref_macrovars_adj<27><<<grd, 128, 0, c->stream>>>(fhat, rhohat, uhat, vhat, what, f, c->rg);
    else k_ref_macrovars_adj<19><<<grd, 128, 0, c->stream>>>(fhat, rhohat, uhat, vhat, what, f, c->rg);
    c->launches++;
    LBM_LAUNCHED(c, "macrovars adjoint");
    return LBM_OK;
}

int lbm_drift_adj(lbm_ctx* c, float* fhat_in, float* fhat_out) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, fhat_in); NEED(c, fhat_out);
    if (fhat_in == fhat_out) return fail(c, LBM_ERR_ARG, "drift_adj: the two adjoint arrays must be distinct");
    const dim3 grd(c->p.ny + 2, c->p.nz + 2);
    if (c->p.nl == 27) k_ref_drift_adj<27><<<grd, 256, 0, c->stream>>>(fhat_in, fhat_out, c->rg);
    else k_ref_drift_adj<19><<<grd, 256, 0, c->stream>>>(fhat_in, fhat_out, c->rg);
    k_ref_zero_interior<<<dim3(c->p.ny, c->p.nz), 256, 0, c->stream>>>(fhat_out, c->rg);
    c->launches += 2;
    LBM_LAUNCHED(c, "drift adjoint");
    return LBM_OK;
}

int lbm_macrovars_drift_adj(lbm_ctx* c, float* fhat_in, float* fhat_out, const float* rhohat, const float* uhat,
                            const float* vhat, const float* what, const float* rho, const float* u, const float* v,
                            const float* w) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, fhat_in); NEED(c, fhat_out); NEED(c, rhohat); NEED(c, uhat); NEED(c, vhat); NEED(c, what);
    NEED(c, rho); NEED(c, u); NEED(c, v); NEED(c, w);
    if (fhat_in == fhat_out) return fail(c, LBM_ERR_ARG, "macrovars_drift_adj: the two adjoint arrays must be distinct");
    const int nl = c->p.nl;
    if (!c->d_adj_terms)
        LBM_TRY(cuda_check(c, cudaMalloc(&c->d_adj_terms, (size_t)4 * c->rg.ncell() * sizeof(float)),
                           "cudaMalloc(macrovars adjoint terms)"));
    k_ref_macro_adj_terms<<<dim3((c->p.nx + 255) / 256, c->p.ny, c->p.nz), 256, 0, c->stream>>>(
        c->d_adj_terms, rhohat, uhat, vhat, what, rho, u, v, w, c->rg);
    const dim3 grd(c->p.ny + 2, c->p.nz + 2);
    if (nl == 27) k_ref_macro_drift_adj<27><<<grd, 256, 0, c->stream>>>(fhat_in, fhat_out, c->d_adj_terms, c->rg);
    else k_ref_macro_drift_adj<19><<<grd, 256, 0, c->stream>>>(fhat_in, fhat_out, c->d_adj_terms, c->rg);
    k_ref_zero_interior<<<dim3(c->p.ny, c->p.nz), 256, 0, c->stream>>>(fhat_out, c->rg);
    c->launches += 3;
    LBM_LAUNCHED(c, "macrovars + drift adjoint");
    return LBM_OK;
}

int lbm_boundarycond_adj(lbm_ctx* c, float* f1hat, float* f2hat, float* uvelhat) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f1hat); NEED(c, f2hat);
    if (c->p.ibnd == 1) NEED(c, uvelhat);
    if (f1hat == f2hat) return fail(c, LBM_ERR_ARG, "boundarycond_adj: f1hat and f2hat must be distinct buffers");
    AdjAcc a1{f1hat, c->rg}, a2{f2hat, c->rg};
    return c->p.nl == 27 ? run_bc_adj<27>(c, a1, a2, uvelhat) : run_bc_adj<19>(c, a1, a2, uvelhat);
}

// ---- the reverse sweep in the state layout --------------------------------------

int lbm_state_bytes(lbm_ctx* c, int64_t* bytes) {
    if (!c || !bytes) return LBM_ERR_ARG;
    *bytes = (int64_t)state_bytes_of(c);
    return LBM_OK;
}

int lbm_state_copy(lbm_ctx* c, void* dst) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, dst);
    if (c->state == ST_NONE) return fail(c, LBM_ERR_STATE, "state_copy: no state imported");
    const size_t n = state_bytes_of(c);
    return cuda_check(c, cudaMemcpyAsync(dst, c->buf[c->cur], n, cudaMemcpyDeviceToDevice, c->stream), "state_copy");
}

static int sadj_check(lbm_ctx* c, const char* what) {
    if (c->p.storage != LBM_STORE_F32) return fail(c, LBM_ERR_UNSUPPORTED, "%s: FP32 state storage only", what);
    if (c->p.ihrr != 1) return fail(c, LBM_ERR_UNSUPPORTED, "%s: the regularized collision (ihrr = 1) only", what);
    if (c->nrturb > 0) return fail(c, LBM_ERR_UNSUPPORTED, "%s: no inflow-turbulence slice", what);
    if (c->force) return fail(c, LBM_ERR_UNSUPPORTED, "%s: no external forcing", what);
    if (c->halo_j) return fail(c, LBM_ERR_UNSUPPORTED, "%s: a whole domain (no j slab)", what);
    return LBM_OK;
}

int lbm_state_adjoint_step(lbm_ctx* c, float* W, float* A, const void* P, int32_t pull, float* uvelhat) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, W); NEED(c, A); NEED(c, P);
    if (c->p.ibnd == 1) NEED(c, uvelhat);
    if (W == A) return fail(c, LBM_ERR_ARG, "state_adjoint_step: W and A must be distinct");
    LBM_TRY(sadj_check(c, "state_adjoint_step"));
    const SoaGrid& g = c->sg;
    const int Q = c->p.nl;
    const int wrap = (c->p.jbnd == 0) ? 1 : 0;   // the stepped state P has no stored j ghost rows
    // The adjoint arrays may read their j ghost rows as rows ny and 1 too, which
    // leaves out the j copies, unless the i and k faces are both closed: then the
    // closed-k kernel reads, through a j ghost row, an x-ghost value of row ny that
    // the closed-i kernel has overwritten since the first j copy.
    const int awrap = (wrap && !(c->face_on[0] && c->face_on[2])) ? 1 : 0;
    const dim3 inner((g.nx + 127) / 128, g.ny, g.nz);
    SoaAdjAcc a1{W, g, awrap}, a2{A, g, awrap};
    if (c->fold && awrap && g.nx >= 2) {
        // inflow/outflow i, periodic j, closed k: the reverse boundary chain is the
        // inflow adjoint then the closed-k adjoint, with the x faces in one kernel
        const unsigned nshell = (unsigned)((sadj_shell_fold_cells(g) + 127) / 128);
        const dim3 xf((g.ny + 31) / 32, Q, g.nz);
        // the launches of a reverse step follow one another with programmatic dependent launch
        if (Q == 27) {
            LBM_TRY(cuda_check(c, launch_pdl(k_sadj_shell_fold<27>, dim3(nshell), dim3(128), c->stream, W, A, g),
                               "state adjoint: shell"));
            LBM_TRY(cuda_check(c, launch_pdl(k_sadj_xface<27>, xf, dim3(32), c->stream, W, A, g, uvelhat, c->p.rho0,
                                             c->cosd, c->sind), "state adjoint: x faces"));
        } else {
            LBM_TRY(cuda_check(c, launch_pdl(k_sadj_shell_fold<19>, dim3(nshell), dim3(128), c->stream, W, A, g),
                               "state adjoint: shell"));
            LBM_TRY(cuda_check(c, launch_pdl(k_sadj_xface<19>, xf, dim3(32), c->stream, W, A, g, uvelhat, c->p.rho0,
                                             c->cosd, c->sind), "state adjoint: x faces"));
        }
        c->launches += 2;
        if (c->face_on[2]) {
            LBM_TRY(cuda_check(c, launch_pdl(k_closed_adj<SoaAdjAcc>, dim3((g.nx + 127) / 128, g.ny, 2), dim3(128),
                                             c->stream, a1, a2, 2, c->face[2][0], c->face[2][1]),
                               "state adjoint: closed k"));
            c->launches++;
        }
        LBM_LAUNCHED(c, "state adjoint: boundaries");
    } else {
        const unsigned shell = (unsigned)((sadj_shell_cells(g, awrap != 0) + 127) / 128);
        if (Q == 27) k_sadj_shell<27><<<shell, 128, 0, c->stream>>>(W, A, g, awrap);
        else k_sadj_shell<19><<<shell, 128, 0, c->stream>>>(W, A, g, awrap);
        c->launches++;
        LBM_LAUNCHED(c, "state adjoint: shell");
        LBM_TRY(Q == 27 ? run_bc_adj<27>(c, a1, a2, uvelhat, awrap != 0)
                        : run_bc_adj<19>(c, a1, a2, uvelhat, awrap != 0));
    }
    const float* Pf = static_cast<const float*>(P);
    const uint8_t* sol = c->d_solid;
    const float* abl = c->d_abl;
    cudaError_t r;
    if (Q == 27)
        r = pull ? launch_pdl(k_sadj_cell<27, true>, inner, dim3(128), c->stream, W, A, Pf, g, wrap, awrap, sol, c->cp, abl)
                 : launch_pdl(k_sadj_cell<27, false>, inner, dim3(128), c->stream, W, A, Pf, g, wrap, awrap, sol, c->cp, abl);
    else
        r = pull ? launch_pdl(k_sadj_cell<19, true>, inner, dim3(128), c->stream, W, A, Pf, g, wrap, awrap, sol, c->cp, abl)
                 : launch_pdl(k_sadj_cell<19, false>, inner, dim3(128), c->stream, W, A, Pf, g, wrap, awrap, sol, c->cp, abl);
    LBM_TRY(cuda_check(c, r, "state adjoint: collision"));
    c->launches++;
    LBM_LAUNCHED(c, "state adjoint: collision");
    return LBM_OK;
}

int lbm_state_adjoint_seed(lbm_ctx* c, float* A, const void* P, const int32_t* probes, const float* uhat,
                           int32_t nprobes) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, A); NEED(c, P); NEED(c, probes); NEED(c, uhat);
    if (nprobes < 1) return fail(c, LBM_ERR_ARG, "state_adjoint_seed: no probes");
    LBM_TRY(sadj_check(c, "state_adjoint_seed"));
    const int wrap = (c->p.jbnd == 0) ? 1 : 0;
    const float* Pf = static_cast<const float*>(P);
    if (c->p.nl == 27) k_sadj_seed<27><<<(nprobes + 127) / 128, 128, 0, c->stream>>>(A, Pf, c->sg, wrap, probes, uhat, nprobes);
    else k_sadj_seed<19><<<(nprobes + 127) / 128, 128, 0, c->stream>>>(A, Pf, c->sg, wrap, probes, uhat, nprobes);
    c->launches++;
    LBM_LAUNCHED(c, "state adjoint: seed");
    return LBM_OK;
}

int lbm_state_adjoint_export(lbm_ctx* c, float* fhat, const float* A) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, fhat); NEED(c, A);
    const SoaGrid& g = c->sg;
    const dim3 all((g.nx + 2 + 127) / 128, g.ny + 2, g.nz + 2);
    if (c->p.nl == 27) k_sadj_export<27><<<all, 128, 0, c->stream>>>(fhat, A, g);
    else k_sadj_export<19><<<all, 128, 0, c->stream>>>(fhat, A, g);
    c->launches++;
    LBM_LAUNCHED(c, "state adjoint: export");
    return LBM_OK;
}

}  // extern "C"
