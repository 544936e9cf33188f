// turbulence_host.cuh -- C ABI of the GPU inflow-turbulence generator
// (declaration in include/lbm_b200.h).  Included at the end of api.cu.

#include <cufft.h>

#include "turbulence.cuh"

extern "C" {

int lbm_inflow_turbulence_compute(lbm_ctx* c, float* uu, float* vv, float* ww, float* rr, int32_t nrturb,
                                  uint64_t seed) {
    if (!c) return LBM_ERR_ARG;
    NEED(c, uu); NEED(c, vv); NEED(c, ww);
    if (nrturb < 1) return fail(c, LBM_ERR_ARG, "inflow_turbulence_compute: nrturb must be positive");
    const int ny = c->p.ny, nz = c->p.nz;
    if ((long long)ny * nz < 2) return fail(c, LBM_ERR_ARG, "inflow_turbulence_compute: the (j, k) plane needs 2 cells");
    // m_inflow_turbulence_compute.F90:19-20, 28-32 and m_pseudo2D.F90:61-105: n1 = ny, n2 = nz made even,
    // dx = dy = 1, decorrelation length 10/sqrt(3) in both directions, theta = 0, no mean
    const int n1 = ny + (ny & 1), n2 = nz + (nz & 1);
    const int nf = rr ? 4 : 3;
    const double pi2 = 2.0 * 3.141592653589793;
    const double rx = 10.0 / sqrt(3.0);
    const double deltak = pi2 * pi2 / ((double)n1 * n2);
    const double kappa2 = (pi2 / n1) * (pi2 / n1), lambda2 = (pi2 / n2) * (pi2 / n2);
    const double r1 = sqrt(8.0) / rx, r2 = sqrt(8.0) / rx;   // the reference derives both from rx
    double summ = 0.0;
    for (int p = -n2 / 2 + 1; p <= n2 / 2; ++p)
        for (int l = -n1 / 2 + 1; l <= n1 / 2; ++l)
            summ += exp(-2.0 * (kappa2 * l * l / (r1 * r1) + lambda2 * p * p / (r2 * r2)));
    summ -= 1.0;   // the mean is not sampled
    const double cc = sqrt(1.0 / (deltak * summ));
    TurbSpec s;
    s.n1 = n1;
    s.n2 = n2;
    s.nb = nf * (nrturb + 1);
    s.amp = (float)(sqrt(deltak) * cc);
    s.ak = (float)(kappa2 / (r1 * r1));
    s.al = (float)(lambda2 / (r2 * r2));
    s.seed = seed;

    int rc = LBM_OK;
    float2* X = nullptr;
    float* Y = nullptr;
    float** outs = nullptr;
    cufftHandle plan = 0;
    bool planned = false;
    const size_t nx_c = (size_t)s.nb * n2 * (n1 / 2 + 1), ny_r = (size_t)s.nb * n2 * n1;
    auto chk = [&](cudaError_t e, const char* w) {
        if (rc == LBM_OK && e != cudaSuccess) rc = cuda_check(c, e, w);
    };
    chk(cudaMalloc(&X, nx_c * sizeof(float2)), "cudaMalloc(turbulence spectrum)");
    chk(cudaMalloc(&Y, ny_r * sizeof(float)), "cudaMalloc(turbulence fields)");
    chk(cudaMalloc(&outs, 4 * sizeof(float*)), "cudaMalloc(turbulence outputs)");
    if (rc == LBM_OK) {
        float* h[4] = {uu, vv, ww, rr};
        chk(cudaMemcpyAsync(outs, h, 4 * sizeof(float*), cudaMemcpyHostToDevice, c->stream), "turbulence outputs");
    }
    if (rc == LBM_OK) {
        int n[2] = {n2, n1};
        if (cufftPlanMany(&plan, 2, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, s.nb) != CUFFT_SUCCESS)
            rc = fail(c, LBM_ERR_CUDA, "inflow_turbulence_compute: cufftPlanMany failed");
        else planned = true;
        if (rc == LBM_OK && cufftSetStream(plan, c->stream) != CUFFT_SUCCESS)
            rc = fail(c, LBM_ERR_CUDA, "inflow_turbulence_compute: cufftSetStream failed");
    }
    if (rc == LBM_OK) {
        k_turb_spectrum<<<(unsigned)((nx_c + 255) / 256), 256, 0, c->stream>>>(X, s);
        c->launches++;
        chk(cudaGetLastError(), "turbulence spectrum");
    }
    if (rc == LBM_OK && cufftExecC2R(plan, reinterpret_cast<cufftComplex*>(X), Y) != CUFFT_SUCCESS)
        rc = fail(c, LBM_ERR_CUDA, "inflow_turbulence_compute: cufftExecC2R failed");
    if (rc == LBM_OK) {
        k_turb_ar1<1024><<<nf, 1024, 0, c->stream>>>(Y, outs, ny, nz, n1, n2, nrturb);
        c->launches++;
        chk(cudaGetLastError(), "turbulence levels");
    }
    // the temporaries are released after the work that uses them
    if (X || Y || outs) chk(cudaStreamSynchronize(c->stream), "inflow_turbulence_compute");
    if (planned) cufftDestroy(plan);
    cudaFree(X);
    cudaFree(Y);
    cudaFree(outs);
    return rc;
}

}  // extern "C"
