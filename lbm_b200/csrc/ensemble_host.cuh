// ensemble_host.cuh -- C ABI of the batched ensemble (declarations in
// include/lbm_b200.h).  Included at the end of api.cu, whose lbm_ctx and
// helpers it uses.
//
// The members are ordinary contexts (lbm_create), so every per-member entry
// point (import, export, set_inflow, set_turbulence, get_macro, ...) applies to
// them.  lbm_ensemble_step advances all of them together: two launches per step
// (k_ens_step, k_ens_bc) on the ensemble's own stream, replayed from a CUDA
// graph of LBM_ENS_GRAPH_STEPS steps when the step count allows.

#include "ensemble.cuh"

namespace {

// launch shapes the autotuner chooses from: threads per block of k_ens_step,
// the minimum resident blocks per SM it is compiled for (its register cap) and
// the tiles of a block's threads each block covers
constexpr int kEnsThreads[LBM_ENS_VARIANTS] = {64, 64, 128, 128, 128, 128, 256, 256};
constexpr int kEnsMinBlocks[LBM_ENS_VARIANTS] = {12, 12, 5, 6, 5, 6, 3, 3};
constexpr int kEnsTiles[LBM_ENS_VARIANTS] = {1, 2, 2, 2, 4, 4, 2, 4};

// why the last lbm_ensemble_create of this thread failed (it returns no handle)
thread_local std::string g_create_err;

}  // namespace

struct lbm_ensemble {
    std::vector<lbm_ctx*> m;
    int nl = 19;
    int storage = LBM_STORE_F32;
    cudaStream_t stream = nullptr;   // own non-blocking stream (graphs cannot capture the legacy stream)
    cudaEvent_t ev[2] = {nullptr, nullptr};
    EnsMember* d_mem = nullptr;
    std::vector<EnsMember> h_mem;
    int2* d_blk = nullptr;           // per block (member, block within member): step grids per variant, then boundaries
    size_t blk_off[LBM_ENS_VARIANTS + 1] = {};
    int nblk[LBM_ENS_VARIANTS + 1] = {};
    int variant = 3;
    int graph_steps = LBM_ENS_GRAPH_STEPS;
    cudaGraphExec_t graph = nullptr;
    int graph_variant = -1;
    int cur = 0;
    std::string err;
};

namespace {

int efail(lbm_ensemble* e, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (e) e->err = buf;
    return code;
}
int echeck(lbm_ensemble* e, cudaError_t r, const char* what) {
    if (r == cudaSuccess) return LBM_OK;
    return efail(e, r == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(r));
}
// a member's error, reported as the ensemble's
int emember(lbm_ensemble* e, int m, int rc) {
    if (rc == LBM_OK) return rc;
    return efail(e, rc, "member %d: %s", m, e->m[m]->err.c_str());
}

EnsLayout ens_layout(const lbm_ensemble* e, int which) {
    EnsLayout L;
    L.mem = e->d_mem;
    L.blk = e->d_blk + e->blk_off[which];
    return L;
}

// descriptors of every member for both parities (the members' settings may have
// changed since the last call)
int ens_upload(lbm_ensemble* e) {
    for (size_t k = 0; k < e->m.size(); ++k) {
        lbm_ctx* c = e->m[k];
        EnsMember& d = e->h_mem[k];
        const int keep = c->cur;
        for (int p = 0; p < 2; ++p) {
            c->cur = p;
            d.a[p] = step_args(c);
        }
        c->cur = keep;
        d.buf[0] = c->buf[0];
        d.buf[1] = c->buf[1];
        d.nface_blocks = bc_fold_face_blocks(c->sg, true);
        d.hp = make_fastdiv((unsigned)(c->sg.nx / 2));
        d.ny = make_fastdiv((unsigned)c->sg.ny);
    }
    return echeck(e, cudaMemcpyAsync(e->d_mem, e->h_mem.data(), e->h_mem.size() * sizeof(EnsMember),
                                     cudaMemcpyHostToDevice, e->stream), "ensemble descriptors");
}

// one batched step: the step kernel, then the boundary kernel; ev (or null): events
// recorded before the step kernel, between the two and after the boundary kernel
template <int Q, typename S>
int ens_launch_step(lbm_ensemble* e, int parity, cudaEvent_t* ev) {
    const EnsLayout Ls = ens_layout(e, e->variant);
    const int nb = e->nblk[e->variant];
    if (ev) LBM_TRY(echeck(e, cudaEventRecord(ev[0], e->stream), "ensemble profile"));
    switch (e->variant) {
        case 0: k_ens_step<Q, S, 64, 12, 1><<<nb, 64, 0, e->stream>>>(Ls, parity); break;
        case 1: k_ens_step<Q, S, 64, 12, 2><<<nb, 64, 0, e->stream>>>(Ls, parity); break;
        case 2: k_ens_step<Q, S, 128, 5, 2><<<nb, 128, 0, e->stream>>>(Ls, parity); break;
        case 3: k_ens_step<Q, S, 128, 6, 2><<<nb, 128, 0, e->stream>>>(Ls, parity); break;
        case 4: k_ens_step<Q, S, 128, 5, 4><<<nb, 128, 0, e->stream>>>(Ls, parity); break;
        case 5: k_ens_step<Q, S, 128, 6, 4><<<nb, 128, 0, e->stream>>>(Ls, parity); break;
        case 6: k_ens_step<Q, S, 256, 3, 2><<<nb, 256, 0, e->stream>>>(Ls, parity); break;
        default: k_ens_step<Q, S, 256, 3, 4><<<nb, 256, 0, e->stream>>>(Ls, parity); break;
    }
    LBM_TRY(echeck(e, cudaGetLastError(), "ensemble step"));
    if (ev) LBM_TRY(echeck(e, cudaEventRecord(ev[1], e->stream), "ensemble profile"));
    k_ens_bc<Q, S><<<e->nblk[LBM_ENS_VARIANTS], 128, 0, e->stream>>>(ens_layout(e, LBM_ENS_VARIANTS), parity);
    LBM_TRY(echeck(e, cudaGetLastError(), "ensemble boundaries"));
    if (ev) LBM_TRY(echeck(e, cudaEventRecord(ev[2], e->stream), "ensemble profile"));
    return LBM_OK;
}

int ens_launch(lbm_ensemble* e, int parity, cudaEvent_t* ev = nullptr) {
    const bool h = e->storage == LBM_STORE_F16;
    if (e->nl == 27) return h ? ens_launch_step<27, __half>(e, parity, ev) : ens_launch_step<27, float>(e, parity, ev);
    return h ? ens_launch_step<19, __half>(e, parity, ev) : ens_launch_step<19, float>(e, parity, ev);
}

int ens_graph(lbm_ensemble* e) {
    if (e->graph && e->graph_variant == e->variant) return LBM_OK;
    if (e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    LBM_TRY(echeck(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal), "graph capture"));
    int rc = LBM_OK;
    for (int s = 0; s < e->graph_steps && rc == LBM_OK; ++s) rc = ens_launch(e, s & 1);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (rc != LBM_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    LBM_TRY(echeck(e, ce, "graph capture"));
    const cudaError_t ie = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    LBM_TRY(echeck(e, ie, "graph instantiate"));
    e->graph_variant = e->variant;
    return LBM_OK;
}

// members still holding an imported (pre-collision) state take their first step
// alone (collide in place); afterwards every member must sit on the same buffer
int ens_align(lbm_ensemble* e, int* used) {
    *used = 0;
    bool pre = false;
    for (size_t k = 0; k < e->m.size(); ++k) {
        lbm_ctx* c = e->m[k];
        if (c->state == ST_NONE) return efail(e, LBM_ERR_STATE, "member %d: no state imported", (int)k);
        if (c->force) return efail(e, LBM_ERR_UNSUPPORTED, "member %d: the ensemble kernels take no external forcing", (int)k);
        if (c->buf[c->cur] != c->own[0] && c->buf[c->cur] != c->own[1])
            return efail(e, LBM_ERR_STATE, "member %d: its state is in a caller's buffer (lbm_step_to); import it again",
                         (int)k);
        own_dst(c);
        if (c->state == ST_PRE) {
            LBM_TRY(emember(e, (int)k, step_dispatch(c)));
            pre = true;
        }
    }
    if (pre) *used = 1;
    for (size_t k = 0; k < e->m.size(); ++k)
        if (e->m[k]->state != ST_POST || e->m[k]->cur != e->m[0]->cur)
            return efail(e, LBM_ERR_STATE, "member %d is not at the same step phase as member 0 "
                         "(import all members, then step them only through the ensemble)", (int)k);
    e->cur = e->m[0]->cur;
    return LBM_OK;
}

// n batched steps on the ensemble stream, ordered after and before the members' stream;
// prof (or null): three events per step (ens_launch_step), direct launches only
int ens_run(lbm_ensemble* e, int n, bool allow_graph, cudaEvent_t* prof = nullptr) {
    cudaStream_t ms = e->m[0]->stream;
    LBM_TRY(echeck(e, cudaEventRecord(e->ev[0], ms), "ensemble order"));
    LBM_TRY(echeck(e, cudaStreamWaitEvent(e->stream, e->ev[0], 0), "ensemble order"));
    LBM_TRY(ens_upload(e));
    int left = n;
    while (left > 0) {
        if (prof) {
            LBM_TRY(ens_launch(e, e->cur, prof + 3 * (n - left)));
            e->cur ^= 1;
            left -= 1;
        } else if (allow_graph && e->graph_steps > 0 && e->cur == 0 && left >= e->graph_steps) {
            LBM_TRY(ens_graph(e));
            LBM_TRY(echeck(e, cudaGraphLaunch(e->graph, e->stream), "graph launch"));
            left -= e->graph_steps;   // an even count: the parity is back to 0
        } else {
            LBM_TRY(ens_launch(e, e->cur));
            e->cur ^= 1;
            left -= 1;
        }
    }
    for (lbm_ctx* c : e->m) {
        c->cur = e->cur;
        c->it += n;
        c->launches += 2LL * n;
    }
    LBM_TRY(echeck(e, cudaEventRecord(e->ev[1], e->stream), "ensemble order"));
    return echeck(e, cudaStreamWaitEvent(ms, e->ev[1], 0), "ensemble order");
}

}  // namespace

extern "C" {

int lbm_ensemble_create(lbm_ensemble** out, const lbm_params* members, int32_t nmembers) {
    if (!out || !members || nmembers < 1) return LBM_ERR_ARG;
    *out = nullptr;
    lbm_ensemble* e = new lbm_ensemble();
    e->nl = members[0].nl;
    e->storage = members[0].storage;
    int rc = LBM_OK;
    for (int k = 0; k < nmembers && rc == LBM_OK; ++k) {
        const lbm_params& p = members[k];
        if (p.nl != e->nl || p.storage != e->storage) {
            rc = efail(e, LBM_ERR_ARG, "member %d: every member needs the same lattice and storage", k);
            break;
        }
        if (!(p.ibnd == 1 && p.jbnd == 0 && (p.kbnd == 11 || p.kbnd == 12 || p.kbnd == 21 || p.kbnd == 22))) {
            rc = efail(e, LBM_ERR_UNSUPPORTED, "member %d: the ensemble runs inflow/outflow i, periodic j, closed k", k);
            break;
        }
        if (p.ihrr != 1 || p.nx % 2 != 0 || p.nx < 4) {
            rc = efail(e, LBM_ERR_UNSUPPORTED, "member %d: the ensemble needs ihrr = 1 and an even nx >= 4", k);
            break;
        }
        lbm_ctx* c = nullptr;
        rc = lbm_create(&c, &p);
        if (rc != LBM_OK) {
            efail(e, rc, "member %d: lbm_create failed (%d)", k, rc);
            break;
        }
        e->m.push_back(c);
    }
    const size_t nm = e->m.size();
    if (rc == LBM_OK) rc = echeck(e, cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    for (int q = 0; q < 2 && rc == LBM_OK; ++q)
        rc = echeck(e, cudaEventCreateWithFlags(&e->ev[q], cudaEventDisableTiming), "cudaEventCreate");
    if (rc == LBM_OK) {
        e->h_mem.resize(nm);
        std::vector<int2> blk;
        for (int v = 0; v <= LBM_ENS_VARIANTS && rc == LBM_OK; ++v) {
            e->blk_off[v] = blk.size();
            for (size_t k = 0; k < nm; ++k) {
                const SoaGrid& g = e->m[k]->sg;
                long long nb;
                if (v < LBM_ENS_VARIANTS) {
                    const long long pairs = (long long)(g.nx / 2) * g.ny * g.nz;
                    if (pairs >= (1LL << 31)) rc = efail(e, LBM_ERR_UNSUPPORTED, "member %d: 2^31 pairs or more", (int)k);
                    const long long per_block = (long long)kEnsThreads[v] * kEnsTiles[v];
                    nb = (pairs + per_block - 1) / per_block;
                } else {
                    // k_bc_fold's grid: k-face blocks, then x-ghost blocks
                    nb = bc_fold_face_blocks(g, true) + bc_fold_xg_blocks(g, e->nl, true);
                }
                for (long long b = 0; b < nb; ++b) blk.push_back(make_int2((int)k, (int)b));
            }
            const long long tot = (long long)(blk.size() - e->blk_off[v]);
            if (tot >= (1LL << 31)) rc = efail(e, LBM_ERR_UNSUPPORTED, "ensemble too large for one launch");
            e->nblk[v] = (int)tot;
        }
        if (rc == LBM_OK) rc = echeck(e, cudaMalloc(&e->d_mem, nm * sizeof(EnsMember)), "cudaMalloc(ensemble)");
        if (rc == LBM_OK) rc = echeck(e, cudaMalloc(&e->d_blk, blk.size() * sizeof(int2)), "cudaMalloc(ensemble)");
        if (rc == LBM_OK)
            rc = echeck(e, cudaMemcpy(e->d_blk, blk.data(), blk.size() * sizeof(int2), cudaMemcpyHostToDevice),
                        "ensemble layout");
    }
    if (rc != LBM_OK) {
        g_create_err = e->err.empty() ? "lbm_ensemble_create failed" : e->err;
        lbm_ensemble_destroy(e);
        return rc;
    }
    g_create_err.clear();
    *out = e;
    return LBM_OK;
}

int lbm_ensemble_destroy(lbm_ensemble* e) {
    if (!e) return LBM_ERR_ARG;
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->graph) cudaGraphExecDestroy(e->graph);
    for (cudaEvent_t v : e->ev)
        if (v) cudaEventDestroy(v);
    if (e->stream) cudaStreamDestroy(e->stream);
    cudaFree(e->d_mem);
    cudaFree(e->d_blk);
    for (lbm_ctx* c : e->m) lbm_destroy(c);
    delete e;
    return LBM_OK;
}

const char* lbm_ensemble_last_error(const lbm_ensemble* e) {
    if (e) return e->err.c_str();
    return g_create_err.empty() ? "null ensemble" : g_create_err.c_str();
}

int lbm_ensemble_size(const lbm_ensemble* e, int32_t* nmembers) {
    if (!e || !nmembers) return LBM_ERR_ARG;
    *nmembers = (int32_t)e->m.size();
    return LBM_OK;
}

int lbm_ensemble_member(lbm_ensemble* e, int32_t m, lbm_ctx** ctx) {
    if (!e || !ctx) return LBM_ERR_ARG;
    if (m < 0 || m >= (int32_t)e->m.size()) return efail(e, LBM_ERR_ARG, "member %d out of range", m);
    *ctx = e->m[m];
    return LBM_OK;
}

int lbm_ensemble_step(lbm_ensemble* e, int32_t nsteps) {
    if (!e || nsteps < 0) return LBM_ERR_ARG;
    if (nsteps == 0) return LBM_OK;
    int used = 0;
    LBM_TRY(ens_align(e, &used));
    return ens_run(e, nsteps - used, true);
}

int lbm_ensemble_set_variant(lbm_ensemble* e, int32_t variant) {
    if (!e) return LBM_ERR_ARG;
    if (variant < 0 || variant >= LBM_ENS_VARIANTS) return efail(e, LBM_ERR_ARG, "variant %d out of range", variant);
    e->variant = variant;
    return LBM_OK;
}

int lbm_ensemble_set_graph(lbm_ensemble* e, int32_t graph_steps) {
    if (!e) return LBM_ERR_ARG;
    if (graph_steps < 0 || graph_steps % 2 != 0)
        return efail(e, LBM_ERR_ARG, "graph_steps must be 0 (no graph) or a positive even count");
    if (graph_steps != e->graph_steps && e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    e->graph_steps = graph_steps;
    return LBM_OK;
}

int lbm_ensemble_profile(lbm_ensemble* e, int32_t nsteps, float* step_kernel_ms, float* boundary_kernel_ms) {
    if (!e || nsteps < 1 || !step_kernel_ms || !boundary_kernel_ms) return LBM_ERR_ARG;
    int used = 0;
    LBM_TRY(ens_align(e, &used));
    std::vector<cudaEvent_t> ev(3 * (size_t)nsteps, nullptr);
    int rc = LBM_OK;
    for (size_t q = 0; q < ev.size() && rc == LBM_OK; ++q) rc = echeck(e, cudaEventCreate(&ev[q]), "cudaEventCreate");
    if (rc == LBM_OK) rc = ens_run(e, nsteps, false, ev.data());
    if (rc == LBM_OK) rc = echeck(e, cudaEventSynchronize(ev.back()), "ensemble profile");
    double ks = 0.0, kb = 0.0;
    for (int s = 0; s < nsteps && rc == LBM_OK; ++s) {
        float a = 0.f, b = 0.f;
        rc = echeck(e, cudaEventElapsedTime(&a, ev[3 * s], ev[3 * s + 1]), "ensemble profile");
        if (rc == LBM_OK) rc = echeck(e, cudaEventElapsedTime(&b, ev[3 * s + 1], ev[3 * s + 2]), "ensemble profile");
        ks += a;
        kb += b;
    }
    for (cudaEvent_t v : ev)
        if (v) cudaEventDestroy(v);
    if (rc == LBM_OK) {
        *step_kernel_ms = (float)(ks / nsteps);
        *boundary_kernel_ms = (float)(kb / nsteps);
    }
    return rc;
}

// mean ms per step of n steps launched as they would be by lbm_ensemble_step
// (graph replay when allowed), timed with events on the ensemble's stream
static int ens_time(lbm_ensemble* e, int n, bool graph, cudaEvent_t t0, cudaEvent_t t1, float* ms) {
    LBM_TRY(echeck(e, cudaEventRecord(t0, e->stream), "autotune"));
    LBM_TRY(ens_run(e, n, graph));
    LBM_TRY(echeck(e, cudaEventRecord(t1, e->stream), "autotune"));
    LBM_TRY(echeck(e, cudaEventSynchronize(t1), "autotune"));
    LBM_TRY(echeck(e, cudaEventElapsedTime(ms, t0, t1), "autotune"));
    *ms /= (float)n;
    return LBM_OK;
}

int lbm_ensemble_autotune(lbm_ensemble* e, int32_t trial_steps, int32_t* variant, float* ms_per_step) {
    if (!e || trial_steps < 1) return LBM_ERR_ARG;
    int used = 0;
    LBM_TRY(ens_align(e, &used));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    LBM_TRY(echeck(e, cudaEventCreate(&t0), "cudaEventCreate"));
    int rc = echeck(e, cudaEventCreate(&t1), "cudaEventCreate");
    // 1. every launch shape, direct launches: one warm-up step, then trial_steps timed
    float best = 0.f;
    int bestv = e->variant;
    for (int v = 0; v < LBM_ENS_VARIANTS && rc == LBM_OK; ++v) {
        e->variant = v;
        float ms = 0.f;
        rc = ens_run(e, 1, false);
        if (rc == LBM_OK) rc = ens_time(e, trial_steps, false, t0, t1, &ms);
        if (rc != LBM_OK) break;
        if (ms_per_step) ms_per_step[v] = ms;
        if (v == 0 || ms < best) {
            best = ms;
            bestv = v;
        }
    }
    e->variant = bestv;
    // 2. the fastest shape replayed from graphs of LBM_ENS_GRAPH_STEPS steps against
    // direct launches, over one graph's worth of steps each (graphs start on parity 0)
    const int g = LBM_ENS_GRAPH_STEPS;
    if (rc == LBM_OK && e->cur != 0) rc = ens_run(e, 1, false);
    if (rc == LBM_OK) {
        e->graph_steps = g;
        rc = ens_run(e, g, true);   // capture and instantiate outside the timing
    }
    float ms_graph = 0.f, ms_direct = 0.f;
    if (rc == LBM_OK) rc = ens_time(e, g, true, t0, t1, &ms_graph);
    if (rc == LBM_OK) rc = ens_time(e, g, false, t0, t1, &ms_direct);
    if (rc == LBM_OK && ms_direct < ms_graph) {
        if (e->graph) cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
        e->graph_steps = 0;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (variant) *variant = bestv;
    return rc;
}

int lbm_ensemble_get_config(const lbm_ensemble* e, int32_t* variant, int32_t* graph_steps) {
    if (!e) return LBM_ERR_ARG;
    if (variant) *variant = e->variant;
    if (graph_steps) *graph_steps = e->graph_steps;
    return LBM_OK;
}

int lbm_ensemble_variant_shape(int32_t variant, int32_t* threads, int32_t* min_blocks, int32_t* tiles) {
    if (variant < 0 || variant >= LBM_ENS_VARIANTS) return LBM_ERR_ARG;
    if (threads) *threads = kEnsThreads[variant];
    if (min_blocks) *min_blocks = kEnsMinBlocks[variant];
    if (tiles) *tiles = kEnsTiles[variant];
    return LBM_OK;
}

}  // extern "C"
