// ref_harness.cu — drives the reference's own CUDA code for parity fixtures.  TEST
// INFRASTRUCTURE ONLY (built into oracle/_ref/, never linked by the engine).
//
// The reference translation unit is #included from its source tree (nothing is copied), so
// its file-local kernels and helpers are callable.  Each entry point runs the reference's own
// steps with the point counts pinned, where its drivers would size them from free memory.
#include "methods_cuda.cu"

#include <cstring>
#include <string>

#include "mcq.h"

static thread_local std::string g_err;

extern "C" const char* mcqref_last_error() { return g_err.c_str(); }

static ModelVariant to_ref_model(const mcq_model& m) {
    switch (m.kind) {
        case MCQ_MODEL_GBM: { GBMParams g; g.S0 = m.S0; g.mu = m.mu; g.sigma = m.sigma; g.T = m.T; return g; }
        case MCQ_MODEL_HESTON: {
            HestonParams h; h.S0 = m.S0; h.mu = m.mu; h.kappa = m.kappa; h.theta = m.theta; h.xi = m.xi;
            h.rho = m.rho; h.v0 = m.v0; h.T = m.T;
            h.L[0][0] = 1.0; h.L[0][1] = 0.0; h.L[1][0] = m.hes_L10; h.L[1][1] = m.hes_L11;
            return h;
        }
        case MCQ_MODEL_DUPIRE: {
            DupireLocalParams d; d.S0 = m.S0; d.mu = m.mu; d.sigma0 = m.sigma0; d.alpha = m.alpha;
            d.beta_d = m.beta_d; d.T = m.T; return d;
        }
        case MCQ_MODEL_MULTI_DUPIRE: {
            MultiDupireParams b; b.n = m.n_assets; b.mu = m.mu; b.sigma0 = m.sigma0; b.alpha = m.alpha;
            b.beta_d = m.beta_d; b.T = m.T; b.uncorrelated = m.uncorrelated || !m.L;
            b.S0.assign(m.S0_vec, m.S0_vec + m.n_assets);
            if (!b.uncorrelated) b.L.assign(m.L, m.L + (size_t)m.n_assets * m.n_assets);
            return b;
        }
    }
    throw std::runtime_error("model kind not in the reference");
}

static PayoffVariant to_ref_payoff(const mcq_payoff& p) {
    switch (p.kind) {
        case MCQ_PAYOFF_EUROPEAN: return European{p.K, p.r, p.T};
        case MCQ_PAYOFF_ASIAN: return Asian{p.K};
        case MCQ_PAYOFF_GEOM_ASIAN: return GeomAsian{p.K};
        case MCQ_PAYOFF_LOOKBACK: return Lookback{p.sigma};
        case MCQ_PAYOFF_BARRIER_UP_OUT: return Barrier{p.K, p.B, p.sigma, p.r, p.T};
        case MCQ_PAYOFF_BASKET: return Basket{p.K, p.r, p.T, p.n_assets};
    }
    throw std::runtime_error("payoff kind not in the reference");
}

// bb_precompute (utils.cpp:54-101) restated here because utils.cpp needs Eigen and C++23.
static BBData bb_tables(int N, double T) {
    BBData bb; bb.N = N; bb.T = T;
    bb.map_idx.assign(N, 0); bb.left_idx.assign(N, 0); bb.right_idx.assign(N, 0);
    bb.weight_left.assign(N, 0.0); bb.weight_right.assign(N, 0.0); bb.std_dev.assign(N, 0.0);
    bb.map_idx[0] = N; bb.std_dev[0] = std::sqrt(T);
    int step = 1, levels = 0;
    for (int t = N; t > 1; t >>= 1) levels++;
    for (int lev = 0; lev < levels; lev++) {
        int np = 1 << lev, stride = N >> lev, half = stride >> 1;
        for (int j = 0; j < np; j++) {
            int L = j * stride, R = (j + 1) * stride, M = L + half;
            double tL = L * T / N, tR = R * T / N, tM = M * T / N;
            bb.map_idx[step] = M; bb.left_idx[step] = L; bb.right_idx[step] = R;
            bb.weight_left[step] = (tR - tM) / (tR - tL);
            bb.weight_right[step] = (tM - tL) / (tR - tL);
            bb.std_dev[step] = std::sqrt((tM - tL) * (tR - tM) / (tR - tL));
            step++;
        }
    }
    return bb;
}

// pca_compute's matrix (utils.cpp:131-167) from the caller (Eigen is absent here).
static PCAData pca_from(int m, double T, const double* Mcol) {
    PCAData p; p.m = m; p.T = T;
    p.M_pca.assign(Mcol, Mcol + (size_t)m * m);
    p.M_pca_f32.resize((size_t)m * m);
    for (size_t i = 0; i < p.M_pca.size(); i++) p.M_pca_f32[i] = (float)p.M_pca[i];
    return p;
}

// The reference's own device functions (curand Sobol32 + hh_scramble), integer output.
__global__ void mcqref_k_u32(const curandDirectionVectors32_t* dirvectors, unsigned salt, int dim0,
                             unsigned offset, unsigned* out, long long total, int chunk) {
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int dim = dim0 + (int)(idx / chunk);
    int p = (int)(idx % chunk);
    unsigned int dv[32];
    for (int i = 0; i < 32; i++) dv[i] = dirvectors[dim].v[i];
    curandStateSobol32_t st;
    curand_init(dv, offset + (unsigned int)p, &st);
    unsigned int raw = curand(&st);
    out[idx] = hh_scramble(raw, splitmix32(salt) ^ (unsigned int)dim);
}

#define HARNESS_TRY try {
#define HARNESS_END return 0; } catch (const std::exception& e) { g_err = e.what(); return 1; }

extern "C" int mcqref_sobol_u32(unsigned salt, int dim0, int nd, unsigned offset, long long n, unsigned* out) {
    HARNESS_TRY
    ensure_sobol_dirvectors_uploaded();
    long long total = (long long)nd * n;
    unsigned* d = nullptr;
    CUDA_CHECK(cudaMalloc(&d, total * sizeof(unsigned)));
    mcqref_k_u32<<<(unsigned)((total + 255) / 256), 256>>>(g_d_sobol_dirvectors, salt, dim0, offset, d, total, (int)n);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaMemcpy(out, d, total * sizeof(unsigned), cudaMemcpyDeviceToHost));
    cudaFree(d);
    HARNESS_END
}

// kernel_gen_hh_scrambled_sobol_normal via gen_scrambled_sobol_normal_replica (dims 0..nd-1).
extern "C" int mcqref_sobol_normal(unsigned salt, int nd, unsigned offset, long long n, float* out) {
    HARNESS_TRY
    float* d = nullptr;
    CUDA_CHECK(cudaMalloc(&d, (size_t)nd * n * sizeof(float)));
    gen_scrambled_sobol_normal_replica(d, nd, n, offset, salt);
    CUDA_CHECK(cudaDeviceSynchronize());
    CUDA_CHECK(cudaMemcpy(out, d, (size_t)nd * n * sizeof(float), cudaMemcpyDeviceToHost));
    cudaFree(d);
    HARNESS_END
}

// accumulate_range (methods_cuda.cu:1549-1622) for R replicas with a pinned point count:
// generate, transform (raw scale / bridge / PCA GEMM), correlate, price, reduce.
// sums[2r], sums[2r+1] = {sum Y, sum Y^2}; *ms = device time of all replicas.
extern "C" int mcqref_qmc_pass(const mcq_model* m, const mcq_payoff* p, int n_steps, int mode,
                               const double* pca_M, unsigned salt0, int R, unsigned offset, long long N,
                               double* sums, float* ms) {
    HARNESS_TRY
    ModelVariant mv = to_ref_model(*m);
    PayoffVariant pv = to_ref_payoff(*p);
    const int d_noise = model_noise_dim(mv);
    const long long D = (long long)n_steps * d_noise;
    const ModelKind mk = model_kind(mv);
    const int pidx = payoff_idx(pv);
    const bool is_multi = (mk == ModelKind::MultiDupire);
    const int n_assets = is_multi ? std::get<MultiDupireParams>(mv).n : 1;
    DeviceBBData* dev_bb = (mode == 1) ? bb_upload(bb_tables(n_steps, model_T(mv))) : nullptr;
    DevicePCAData* dev_pca = (mode == 2) ? pca_upload(pca_from(n_steps, model_T(mv), pca_M)) : nullptr;
    cublasHandle_t cublas = nullptr;
    if (mode == 2 || is_multi) CUBLAS_CHECK(cublasCreate(&cublas));
    DeviceMultiData dm;
    if (is_multi) dm = multi_upload(std::get<MultiDupireParams>(mv));
    float *d_Z = nullptr, *d_dW = nullptr, *d_W = nullptr, *d_corr = nullptr;
    __half* d_Zh = nullptr;
    double* d_sums = nullptr;
    CUDA_CHECK(cudaMalloc(&d_Z, (D * N + 2) * sizeof(float)));
    CUDA_CHECK(cudaMalloc(&d_dW, D * N * sizeof(float)));
    if (mode == 1) CUDA_CHECK(cudaMalloc(&d_W, (n_steps + 1) * N * sizeof(float)));
    if (mode == 2) CUDA_CHECK(cudaMalloc(&d_Zh, D * N * sizeof(__half)));
    if (is_multi && dm.d_L) CUDA_CHECK(cudaMalloc(&d_corr, D * N * sizeof(float)));
    CUDA_CHECK(cudaMalloc(&d_sums, 4 * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    float total_ms = 0.f;
    for (int r = 0; r < R; r++) {
        CUDA_CHECK(cudaMemset(d_sums, 0, 4 * sizeof(double)));
        KernelParams kp = make_params(mv, pv, n_steps);
        CUDA_CHECK(cudaMemcpyToSymbol(c_p, &kp, sizeof(kp)));
        CUDA_CHECK(cudaDeviceSynchronize());
        cudaEventRecord(e0);
        gen_scrambled_sobol_normal_replica(d_Z, D, N, offset, salt0 + (unsigned)r);
        if (mode == 1) {
            CUDA_CHECK(cudaMemset(d_W, 0, (n_steps + 1) * N * sizeof(float)));
            kernel_bb_transform<<<(int)((N + BLOCK_SIZE - 1) / BLOCK_SIZE), BLOCK_SIZE>>>(
                d_Z, d_dW, d_W, dev_bb->d_map_idx, dev_bb->d_left_idx, dev_bb->d_right_idx,
                dev_bb->d_wl, dev_bb->d_wr, dev_bb->d_std_dev, n_steps, (int)N);
        } else if (mode == 2) {
            kernel_cast_f32_to_f16<<<(int)((D * N + BLOCK_SIZE - 1) / BLOCK_SIZE), BLOCK_SIZE>>>(d_Z, d_Zh, (int)(D * N));
            phase1_pca(cublas, dev_pca->d_M_pca_f16, d_Zh, d_dW, (int)D, (int)N);
        } else {
            CUDA_CHECK(cudaMemcpy(d_dW, d_Z, D * N * sizeof(float), cudaMemcpyDeviceToDevice));
            kernel_scale<<<(int)((D * N + BLOCK_SIZE - 1) / BLOCK_SIZE), BLOCK_SIZE>>>(d_dW, sqrtf(kp.h), D * N);
        }
        const float* feed = d_dW;
        if (is_multi && dm.d_L) {
            correlate_multi_dupire(cublas, dm, d_dW, d_corr, n_steps, (int)N);
            feed = d_corr;
        }
        launch_mc_kernel(mk, pidx, is_multi, feed, d_sums, (int)N, n_steps, n_assets, dm.d_S0);
        cudaEventRecord(e1);
        CUDA_CHECK(cudaDeviceSynchronize());
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        total_ms += t;
        double hs[4];
        CUDA_CHECK(cudaMemcpy(hs, d_sums, 4 * sizeof(double), cudaMemcpyDeviceToHost));
        sums[2 * r] = hs[0];
        sums[2 * r + 1] = hs[1];
    }
    if (ms) *ms = total_ms;
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaFree(d_Z); cudaFree(d_dW); cudaFree(d_W); cudaFree(d_Zh); cudaFree(d_corr); cudaFree(d_sums);
    if (is_multi) multi_free(dm);
    if (cublas) cublasDestroy(cublas);
    if (dev_bb) bb_free(dev_bb);
    if (dev_pca) pca_free(dev_pca);
    HARNESS_END
}

// kernel_mlmc (methods_cuda.cu:445-518) as run_mlqmc_cuda's launch_level runs one level in raw
// mode (:1849-1919), with the point count pinned: per replica, scrambled Sobol normals for salt
// salt0 + r from point `offset`, kernel_scale by sqrt(h_fine) (not for Heston, which scales
// inside), then the level kernel.  level0 != 0: no coarse path (N_coarse = 0, as level 0).
// sums[4r .. 4r + 3] = {sum dY, sum dY^2, sum Yf, sum Yf^2}.
extern "C" int mcqref_level_pass(const mcq_model* m, const mcq_payoff* p, int n_fine, int M, int level0,
                                 unsigned salt0, int R, unsigned offset, long long N, double* sums) {
    HARNESS_TRY
    ModelVariant mv = to_ref_model(*m);
    PayoffVariant pv = to_ref_payoff(*p);
    const ModelKind mk = model_kind(mv);
    const int pidx = payoff_idx(pv);
    if (mk == ModelKind::MultiDupire) throw std::runtime_error("the reference has no multi-asset level kernel");
    KernelParams kp = make_params(mv, pv, 1);   // as run_mlqmc_cuda, :1720-1722
    kp.M_refine = M;
    CUDA_CHECK(cudaMemcpyToSymbol(c_p, &kp, sizeof(kp)));
    const double T = model_T(mv);
    const int N_fine = n_fine, N_coarse = level0 ? 0 : n_fine / M;
    const float h_fine = (float)(T / N_fine), h_coarse = (float)(T / std::max(N_coarse, 1));
    const float sqrt_hf = sqrtf(h_fine);
    const long long D = (long long)N_fine * model_noise_dim(mv);
    const long long gen_count = (D * N + 1) & ~1LL;
    float* d_Z = nullptr;
    double* d_sums = nullptr;
    CUDA_CHECK(cudaMalloc(&d_Z, (D * N + 2) * sizeof(float)));
    CUDA_CHECK(cudaMalloc(&d_sums, 4 * sizeof(double)));
    for (int r = 0; r < R; r++) {
        CUDA_CHECK(cudaMemset(d_sums, 0, 4 * sizeof(double)));
        gen_scrambled_sobol_normal_replica(d_Z, D, N, offset, salt0 + (unsigned)r);
        if (mk != ModelKind::Heston)
            kernel_scale<<<(int)((gen_count + BLOCK_SIZE - 1) / BLOCK_SIZE), BLOCK_SIZE>>>(d_Z, sqrt_hf, gen_count);
        MLMC_TABLE[(int)mk][pidx]<<<(int)((N + BLOCK_SIZE - 1) / BLOCK_SIZE), BLOCK_SIZE>>>(
            d_Z, d_sums, (int)N, N_fine, N_coarse, M, h_fine, h_coarse, sqrt_hf);
        CUDA_CHECK(cudaGetLastError());
        CUDA_CHECK(cudaDeviceSynchronize());
        CUDA_CHECK(cudaMemcpy(sums + 4 * r, d_sums, 4 * sizeof(double), cudaMemcpyDeviceToHost));
    }
    cudaFree(d_Z); cudaFree(d_sums);
    HARNESS_END
}

// kernel_is_gbm (methods_cuda.cu:685-707) with the parameters run_is_cuda sets (:2288-2298) and
// scrambled Sobol normals (salt salt0 + r, from point `offset`) in place of its XORWOW stream;
// z_star_step is the per-step shift.  sums[2r], sums[2r + 1] = {sum Y, sum Y^2}.
extern "C" int mcqref_is_pass(const mcq_model* m, const mcq_payoff* p, int n_steps, double z_star_step,
                              unsigned salt0, int R, unsigned offset, long long N, double* sums) {
    HARNESS_TRY
    if (m->kind != MCQ_MODEL_GBM || p->kind != MCQ_PAYOFF_EUROPEAN) throw std::runtime_error("IS: GBM European");
    KernelParams kp{};
    kp.S0 = (float)m->S0; kp.mu = (float)m->mu; kp.sigma = (float)m->sigma; kp.T = (float)m->T;
    kp.K = (float)p->K; kp.r = (float)p->r;
    kp.discount = (float)std::exp(-p->r * p->T);
    kp.payoff_kind = PayoffKind::European;
    kp.z_star = (float)z_star_step;
    kp.h = kp.T / n_steps;
    CUDA_CHECK(cudaMemcpyToSymbol(c_p, &kp, sizeof(kp)));
    float* d_Z = nullptr;
    double* d_sums = nullptr;
    CUDA_CHECK(cudaMalloc(&d_Z, ((long long)n_steps * N + 2) * sizeof(float)));
    CUDA_CHECK(cudaMalloc(&d_sums, 4 * sizeof(double)));
    for (int r = 0; r < R; r++) {
        CUDA_CHECK(cudaMemset(d_sums, 0, 4 * sizeof(double)));
        gen_scrambled_sobol_normal_replica(d_Z, n_steps, N, offset, salt0 + (unsigned)r);
        kernel_is_gbm<<<(int)((N + BLOCK_SIZE - 1) / BLOCK_SIZE), BLOCK_SIZE>>>(d_Z, d_sums, (int)N, n_steps);
        CUDA_CHECK(cudaGetLastError());
        CUDA_CHECK(cudaDeviceSynchronize());
        double hs[4];
        CUDA_CHECK(cudaMemcpy(hs, d_sums, 4 * sizeof(double), cudaMemcpyDeviceToHost));
        sums[2 * r] = hs[0];
        sums[2 * r + 1] = hs[1];
    }
    cudaFree(d_Z); cudaFree(d_sums);
    HARNESS_END
}

// The reference's adaptive drivers, unmodified, for statistical comparison.
extern "C" int mcqref_run_mlqmc(const mcq_model* m, const mcq_payoff* p, double eps, int M, int max_L,
                                int pilot_n, int R, double* out4) {
    HARNESS_TRY
    MLMCConfig ml; ml.M = M; ml.max_L = max_L; ml.pilot_n = pilot_n;
    QMCConfig qc; qc.R = R;
    MCResult r = run_mlqmc_cuda(to_ref_model(*m), to_ref_payoff(*p), eps, ml, qc, NoiseMode::Raw);
    out4[0] = r.price; out4[1] = r.std_error; out4[2] = (double)r.n_samples; out4[3] = r.time_s;
    HARNESS_END
}

extern "C" int mcqref_run_mlmc(const mcq_model* m, const mcq_payoff* p, double eps, int M, int max_L,
                               int pilot_n, double* out4) {
    HARNESS_TRY
    MLMCConfig ml; ml.M = M; ml.max_L = max_L; ml.pilot_n = pilot_n;
    MCResult r = run_mlmc_cuda(to_ref_model(*m), to_ref_payoff(*p), eps, ml);
    out4[0] = r.price; out4[1] = r.std_error; out4[2] = (double)r.n_samples; out4[3] = r.time_s;
    HARNESS_END
}

extern "C" int mcqref_run_mc(const mcq_model* m, const mcq_payoff* p, double eps, int n_steps, double* out4) {
    HARNESS_TRY
    MCConfig c;
    MCResult r = run_mc_cuda(to_ref_model(*m), to_ref_payoff(*p), eps, n_steps, c);
    out4[0] = r.price; out4[1] = r.std_error; out4[2] = (double)r.n_samples; out4[3] = r.time_s;
    HARNESS_END
}
