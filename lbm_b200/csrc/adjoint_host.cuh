// adjoint_host.cuh -- C ABI of the adjoint kernels (declarations in
// include/lbm_b200.h).  Included at the end of api.cu, whose lbm_ctx and
// boundary tables it uses.

#include "adjoint.cuh"

namespace {

// boundarycond in reverse: the launches of run_bc in the opposite order, each
// with the adjoint accessor (a copy becomes an accumulation into its source)
template <int Q>
int run_bc_adj(lbm_ctx* c, float* f1h, float* f2h, float* uvelh) {
    const int nx = c->p.nx, ny = c->p.ny, nz = c->p.nz, nl = c->p.nl;
    cudaStream_t s = c->stream;
    AdjAcc a1{f1h, c->rg}, a2{f2h, c->rg};
    auto periodic = [&](int axis) {
        dim3 grd;
        if (axis == 0) grd = dim3((ny + 2 + 127) / 128, nz + 2, nl);
        else if (axis == 1) grd = dim3((nx + 2 + 127) / 128, nz + 2, nl);
        else grd = dim3((nx + 2 + 127) / 128, ny + 2, nl);
        k_periodic<AdjAcc><<<grd, 128, 0, s>>>(a1, axis, nl);
        c->launches++;
    };
    const int codes[3] = {c->p.ibnd, c->p.jbnd, c->p.kbnd};
    for (int a = 2; a >= 0; --a)
        if (codes[a] == 0) periodic(a);
    if (c->p.ibnd == 1) {
        k_inflow_adj<Q><<<dim3((ny + 127) / 128, nz), 128, 0, s>>>(a1, uvelh, c->p.rho0, c->cosd, c->sind);
        c->launches++;
    }
    if (c->corners_on) {
        k_corners<AdjAcc><<<1, 32, 0, s>>>(a1, a2, c->corners);
        c->launches++;
    }
    for (int e = 2; e >= 0; --e) {
        if (!c->edges_on[e]) continue;
        const EdgeSet& es = c->edges[e];
        k_edges<AdjAcc><<<dim3((es.nfree + 127) / 128, 4), 128, 0, s>>>(a1, a2, es);
        c->launches++;
    }
    for (int a = 2; a >= 0; --a) {
        if (!c->face_on[a]) continue;
        const int na = (a == 0) ? ny : nx;
        const int nb = (a == 2) ? ny : nz;
        k_closed<AdjAcc><<<dim3((na + 127) / 128, nb, 2), 128, 0, s>>>(a1, a2, a, c->face[a][0], c->face[a][1], 1, 1);
        c->launches++;
    }
    for (int a = 2; a >= 0; --a)
        if (codes[a] == 0) periodic(a);
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
    const int nl = c->p.nl;
    k_ref_drift_adj<<<dim3((nl * (c->p.nx + 2) + 127) / 128, c->p.ny + 2, c->p.nz + 2), 128, 0, c->stream>>>(
        fhat_in, fhat_out, c->rg);
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
    const dim3 grd(c->p.ny + 2, c->p.nz + 2);
    if (nl == 27)
        k_ref_macro_drift_adj<27><<<grd, 256, 0, c->stream>>>(fhat_in, fhat_out, rhohat, uhat, vhat, what, rho, u, v, w,
                                                             c->rg);
    else
        k_ref_macro_drift_adj<19><<<grd, 256, 0, c->stream>>>(fhat_in, fhat_out, rhohat, uhat, vhat, what, rho, u, v, w,
                                                             c->rg);
    k_ref_zero_interior<<<dim3(c->p.ny, c->p.nz), 256, 0, c->stream>>>(fhat_out, c->rg);
    c->launches += 2;
    LBM_LAUNCHED(c, "macrovars + drift adjoint");
    return LBM_OK;
}

int lbm_boundarycond_adj(lbm_ctx* c, float* f1hat, float* f2hat, float* uvelhat) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, f1hat); NEED(c, f2hat);
    if (c->p.ibnd == 1) NEED(c, uvelhat);
    if (f1hat == f2hat) return fail(c, LBM_ERR_ARG, "boundarycond_adj: f1hat and f2hat must be distinct buffers");
    return c->p.nl == 27 ? run_bc_adj<27>(c, f1hat, f2hat, uvelhat) : run_bc_adj<19>(c, f1hat, f2hat, uvelhat);
}

}  // extern "C"
