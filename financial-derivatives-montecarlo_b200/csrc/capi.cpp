// capi.cpp — the extern "C" boundary (include/mcq.h).  Every entry point takes the engine lock,
// makes sure the device context exists, converts C++ exceptions into status codes and records
// the message for mcq_last_error().
#include <cuda_fp16.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "book.h"
#include "drivers.h"
#include "support.h"

using namespace mcq;

static thread_local std::string g_last_error;

namespace mcq {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace mcq

#define API_BEGIN                                   \
    try {                                           \
        std::lock_guard<std::mutex> lk_(engine().mu);
#define API_BEGIN_NOINIT \
    try {                \
        std::lock_guard<std::mutex> lk_(engine().mu);
#define API_END                                      \
    return MCQ_OK;                                   \
    }                                                \
    catch (const Error& e) {                         \
        g_last_error = e.what();                     \
        return e.code;                               \
    }                                                \
    catch (const std::bad_alloc&) {                  \
        g_last_error = "host allocation failed";     \
        return MCQ_ERR_NOMEM;                        \
    }                                                \
    catch (const std::exception& e) {                \
        g_last_error = e.what();                     \
        return MCQ_ERR_INTERNAL;                     \
    }                                                \
    catch (...) {                                    \
        g_last_error = "unknown error";              \
        return MCQ_ERR_INTERNAL;                     \
    }

#define NEED(ptr) MCQ_REQUIRE((ptr) != nullptr, MCQ_ERR_INVALID, #ptr " is NULL")

static const Handle* as_handle(mcq_handle h, int kind) {
    if (!h) return nullptr;
    const Handle* H = reinterpret_cast<const Handle*>(h);
    MCQ_REQUIRE(H->kind == kind, MCQ_ERR_INVALID, "handle of the wrong kind");
    return H;
}

extern "C" {

const char* mcq_last_error(void) { return g_last_error.c_str(); }
int mcq_version(void) { return 100; }

int mcq_init(int device) {
    API_BEGIN_NOINIT
    ensure_ready(device);
    API_END
}

int mcq_shutdown(void) {
    API_BEGIN_NOINIT
    shutdown_engine();
    API_END
}

int mcq_default_cfgs(mcq_mc_cfg* mc, mcq_qmc_cfg* qmc, mcq_mlmc_cfg* ml) {
    if (mc) { mc->N_batch = 1LL << 16; mc->pilot_n = 10000; mc->seed = 123u; }        // methods_cuda.cuh:10-14
    if (qmc) { qmc->R = 32; qmc->max_doublings = 20; qmc->N0_per_replica = 0; qmc->salt_base = 42u; qmc->flags = 0; }
    if (ml) { ml->M = 2; ml->max_L = 10; ml->pilot_n = 400; ml->n0_steps = 1; ml->flags = 0; ml->seed = 42u; }
    return MCQ_OK;
}

int mcq_model_heston(double S0, double mu, double kappa, double theta, double xi, double rho,
                     double v0, double T, mcq_model* out) {
    if (!out) { g_last_error = "out is NULL"; return MCQ_ERR_INVALID; }
    std::memset(out, 0, sizeof(*out));
    out->kind = MCQ_MODEL_HESTON;
    out->S0 = S0; out->mu = mu; out->kappa = kappa; out->theta = theta; out->xi = xi;
    out->rho = rho; out->v0 = v0; out->T = T;
    out->hes_L10 = rho;                          // HestonParams::compute_cholesky, models.hpp:36-42
    out->hes_L11 = std::sqrt(1.0 - rho * rho);
    return MCQ_OK;
}

// ------------------------------------------------------------------ BB / PCA handles

int mcq_bb_create(int N, double T, mcq_handle* out) {
    API_BEGIN
    NEED(out);
    MCQ_REQUIRE(N > 0 && (N & (N - 1)) == 0 && N <= 4096, MCQ_ERR_INVALID, "BB needs N a power of two <= 4096");
    MCQ_REQUIRE(T > 0, MCQ_ERR_INVALID, "BB needs T > 0");
    // bb_precompute (utils.cpp:54-101): step 0 is W[N]; then level-order midpoints.
    std::vector<int> map(N, 0), left(N, 0), right(N, 0);
    std::vector<double> wl(N, 0.0), wr(N, 0.0), sd(N, 0.0);
    map[0] = N;
    sd[0] = std::sqrt(T);
    int step = 1, levels = 0;
    for (int t = N; t > 1; t >>= 1) levels++;
    for (int lev = 0; lev < levels; lev++) {
        const int np = 1 << lev, stride = N >> lev, half = stride >> 1;
        for (int j = 0; j < np; j++) {
            const int L = j * stride, R = (j + 1) * stride, M = L + half;
            const double tL = L * T / N, tR = R * T / N, tM = M * T / N;
            map[step] = M; left[step] = L; right[step] = R;
            wl[step] = (tR - tM) / (tR - tL);
            wr[step] = (tM - tL) / (tR - tL);
            sd[step] = std::sqrt((tM - tL) * (tR - tM) / (tR - tL));
            step++;
        }
    }
    ensure_ready();
    auto* H = new Handle();
    H->kind = MCQ_NOISE_BB;
    H->n = N;
    H->T = T;
    std::vector<float4> w4(N);
    std::vector<int2> lr(N);
    H->host_f.resize((size_t)3 * N);
    H->host_i.resize(N);
    for (int j = 0; j < N; j++) {   // weights uploaded as float, as bb_upload (methods_cuda.cu:944-951)
        float m_bits;
        std::memcpy(&m_bits, &map[j], sizeof(float));
        w4[j] = make_float4((float)wl[j], (float)wr[j], (float)sd[j], m_bits);
        lr[j] = make_int2(left[j], right[j]);
        H->host_f[3 * j] = (float)wl[j];
        H->host_f[3 * j + 1] = (float)wr[j];
        H->host_f[3 * j + 2] = (float)sd[j];
        H->host_i[j] = map[j];
    }
    if (N > 32) {   // window levels of the fused bridge (bb_window): are their weights uniform?
        const int S = N >> 5;
        bool uni = true;
        for (int u = 0; u < 5 && uni; u++) {
            const int d0 = S << u;
            for (int c = 0; c < 3; c++) H->bb_lvl[u][c] = H->host_f[3 * d0 + c];
            for (int q = 0; q < S && uni; q++)
                for (int v = 0; v < (1 << u) && uni; v++) {
                    const int d = (S << u) + (q << u) + v;
                    for (int c = 0; c < 3; c++)
                        if (std::memcmp(&H->host_f[3 * d + c], &H->bb_lvl[u][c], sizeof(float)) != 0) uni = false;
                }
        }
        H->bb_uni = uni;
    }
    try {
        char* d = (char*)H->table.ensure(sizeof(float4) * N + sizeof(int2) * N);
        MCQ_CUDA(cudaMemcpy(d, w4.data(), sizeof(float4) * N, cudaMemcpyHostToDevice));
        MCQ_CUDA(cudaMemcpy(d + sizeof(float4) * N, lr.data(), sizeof(int2) * N, cudaMemcpyHostToDevice));
    } catch (...) {
        delete H;
        throw;
    }
    *out = reinterpret_cast<mcq_handle>(H);
    API_END
}

static void pca_upload_into(Handle* H, int m, const std::vector<double>& M) {
    // fp16 copy, row-major by output step i: row i = M[i][0..m-1] (pca_upload casts to half,
    // methods_cuda.cu:962-971)
    std::vector<__half> hf((size_t)m * m);
    H->host_f.resize((size_t)m * m);
    for (int i = 0; i < m; i++)
        for (int k = 0; k < m; k++) {
            const float f = (float)M[(size_t)k * m + i];
            hf[(size_t)i * m + k] = __float2half(f);
            H->host_f[(size_t)k * m + i] = f;
        }
    void* d = H->table.ensure(sizeof(__half) * (size_t)m * m);
    MCQ_CUDA(cudaMemcpy(d, hf.data(), sizeof(__half) * (size_t)m * m, cudaMemcpyHostToDevice));
}

int mcq_pca_create(int m, double T, mcq_handle* out) {
    API_BEGIN
    NEED(out);
    MCQ_REQUIRE(m >= 1 && m <= 4096 && T > 0, MCQ_ERR_INVALID, "PCA needs 1 <= m <= 4096 and T > 0");
    // pca_compute (utils.cpp:131-167): eigenpairs of C_ij = h min(i+1, j+1) in closed form,
    // descending, sign fixed by a positive first component; M_pca = row-difference of V sqrt(L).
    std::vector<double> M((size_t)m * m);
    const double h = T / m, den = 2.0 * m + 1.0;
    for (int k = 0; k < m; k++) {
        const double s = std::sin((2.0 * k + 1.0) * M_PI / (2.0 * den));
        const double sl = std::sqrt(h / (4.0 * s * s)), c = 2.0 / std::sqrt(den);
        double prev = 0.0;
        for (int i = 0; i < m; i++) {
            const double cum = c * std::sin((2.0 * k + 1.0) * (i + 1.0) * M_PI / den) * sl;
            M[(size_t)k * m + i] = cum - prev;
            prev = cum;
        }
    }
    ensure_ready();
    auto* H = new Handle();
    H->kind = MCQ_NOISE_PCA;
    H->n = m;
    H->T = T;
    try { pca_upload_into(H, m, M); } catch (...) { delete H; throw; }
    *out = reinterpret_cast<mcq_handle>(H);
    API_END
}

int mcq_pca_create_from(int m, double T, const double* Mc, mcq_handle* out) {
    API_BEGIN
    NEED(out); NEED(Mc);
    MCQ_REQUIRE(m >= 1 && m <= 4096, MCQ_ERR_INVALID, "PCA needs 1 <= m <= 4096");
    std::vector<double> M(Mc, Mc + (size_t)m * m);
    ensure_ready();
    auto* H = new Handle();
    H->kind = MCQ_NOISE_PCA;
    H->n = m;
    H->T = T;
    try { pca_upload_into(H, m, M); } catch (...) { delete H; throw; }
    *out = reinterpret_cast<mcq_handle>(H);
    API_END
}

int mcq_handle_free(mcq_handle h) {
    API_BEGIN_NOINIT
    if (h) {
        Handle* H = reinterpret_cast<Handle*>(h);
        MCQ_REQUIRE(H->kind == MCQ_NOISE_BB || H->kind == MCQ_NOISE_PCA, MCQ_ERR_INVALID, "not an mcq handle");
        if (engine().ready) cudaDeviceSynchronize();
        H->kind = -1;
        delete H;
    }
    API_END
}

int mcq_handle_info(mcq_handle h, int* kind, int* n) {
    API_BEGIN_NOINIT
    NEED(h);
    const Handle* H = reinterpret_cast<const Handle*>(h);
    if (kind) *kind = H->kind;
    if (n) *n = H->n;
    API_END
}

int mcq_bb_tables(mcq_handle bb, int* map_idx, float* wl, float* wr, float* sd) {
    API_BEGIN_NOINIT
    const Handle* H = as_handle(bb, MCQ_NOISE_BB);
    NEED(H);
    for (int j = 0; j < H->n; j++) {
        if (map_idx) map_idx[j] = H->host_i[j];
        if (wl) wl[j] = H->host_f[3 * j];
        if (wr) wr[j] = H->host_f[3 * j + 1];
        if (sd) sd[j] = H->host_f[3 * j + 2];
    }
    API_END
}

int mcq_pca_matrix(mcq_handle pca, float* M) {
    API_BEGIN_NOINIT
    const Handle* H = as_handle(pca, MCQ_NOISE_PCA);
    NEED(H); NEED(M);
    std::memcpy(M, H->host_f.data(), sizeof(float) * H->host_f.size());
    API_END
}

// ------------------------------------------------------------------ drivers

int mcq_run_mc(const mcq_model* m, const mcq_payoff* p, double eps, int n_steps,
               const mcq_mc_cfg* cfg, mcq_result* out) {
    API_BEGIN
    NEED(m); NEED(p); NEED(cfg); NEED(out);
    ensure_ready();
    run_mc(*m, *p, eps, n_steps, *cfg, *out);
    API_END
}

int mcq_run_mc_fixed(const mcq_model* m, const mcq_payoff* p, int n_steps, int64_t n_paths,
                     uint32_t seed, double* mean, double* var_of_mean) {
    API_BEGIN
    NEED(m); NEED(p); NEED(mean); NEED(var_of_mean);
    ensure_ready();
    run_mc_fixed(*m, *p, n_steps, n_paths, seed, *mean, *var_of_mean);
    API_END
}

int mcq_run_qmc(const mcq_model* m, const mcq_payoff* p, double eps, int n_steps,
                const mcq_qmc_cfg* cfg, int noise_mode, mcq_handle bb, mcq_handle pca,
                mcq_result* out) {
    API_BEGIN
    NEED(m); NEED(p); NEED(cfg); NEED(out);
    MCQ_REQUIRE(noise_mode >= 0 && noise_mode <= 2, MCQ_ERR_INVALID, "bad noise mode");
    ensure_ready();
    run_qmc(*m, *p, eps, n_steps, *cfg, noise_mode, as_handle(bb, MCQ_NOISE_BB),
            as_handle(pca, MCQ_NOISE_PCA), *out);
    API_END
}

int mcq_run_mlmc(const mcq_model* m, const mcq_payoff* p, double eps, const mcq_mlmc_cfg* cfg,
                 mcq_result* out) {
    API_BEGIN
    NEED(m); NEED(p); NEED(cfg); NEED(out);
    ensure_ready();
    run_mlmc(*m, *p, eps, *cfg, *out);
    API_END
}

int mcq_run_mlqmc(const mcq_model* m, const mcq_payoff* p, double eps, const mcq_mlmc_cfg* ml,
                  const mcq_qmc_cfg* qmc, int noise_mode, const mcq_handle* bb_list, int n_bb,
                  const mcq_handle* pca_list, int n_pca, mcq_result* out) {
    API_BEGIN
    NEED(m); NEED(p); NEED(ml); NEED(qmc); NEED(out);
    MCQ_REQUIRE(noise_mode >= 0 && noise_mode <= 2, MCQ_ERR_INVALID, "bad noise mode");
    std::vector<const Handle*> bl, pl;
    for (int i = 0; i < n_bb; i++) bl.push_back(bb_list ? as_handle(bb_list[i], MCQ_NOISE_BB) : nullptr);
    for (int i = 0; i < n_pca; i++) pl.push_back(pca_list ? as_handle(pca_list[i], MCQ_NOISE_PCA) : nullptr);
    ensure_ready();
    run_mlqmc(*m, *p, eps, *ml, *qmc, noise_mode, bl, pl, *out);
    API_END
}

int mcq_cv_pilot(const mcq_model* main_m, const mcq_model* ctrl_m, const mcq_payoff* main_p,
                 const mcq_payoff* ctrl_p, double E_ctrl, int n_steps, int N_pilot, uint32_t seed,
                 mcq_cv_pilot_out* out) {
    API_BEGIN
    NEED(main_m); NEED(main_p); NEED(out);
    (void)ctrl_m; (void)ctrl_p;   // the reference's CV kernels fix the control (methods_cuda.cu:601-677)
    ensure_ready();
    cv_pilot(*main_m, *main_p, E_ctrl, n_steps, N_pilot, seed, *out);
    API_END
}

int mcq_run_mc_cv(const mcq_model* main_m, const mcq_model* ctrl_m, const mcq_payoff* main_p,
                  const mcq_payoff* ctrl_p, double E_ctrl, double beta, double eps, int n_steps,
                  const mcq_mc_cfg* cfg, mcq_result* out) {
    API_BEGIN
    NEED(main_m); NEED(main_p); NEED(cfg); NEED(out);
    (void)ctrl_m; (void)ctrl_p;
    ensure_ready();
    run_mc_cv(*main_m, *main_p, E_ctrl, beta, eps, n_steps, *cfg, *out);
    API_END
}

int mcq_run_qmc_cv(const mcq_model* main_m, const mcq_model* ctrl_m, const mcq_payoff* main_p,
                   const mcq_payoff* ctrl_p, double E_ctrl, double beta, double eps, int n_steps,
                   const mcq_qmc_cfg* cfg, mcq_result* out) {
    API_BEGIN
    NEED(main_m); NEED(main_p); NEED(cfg); NEED(out);
    (void)ctrl_m; (void)ctrl_p;
    ensure_ready();
    run_qmc_cv(*main_m, *main_p, E_ctrl, beta, eps, n_steps, *cfg, *out);
    API_END
}

int mcq_run_is(const mcq_model* gbm, const mcq_payoff* european, double z_star, double eps,
               const mcq_mc_cfg* cfg, mcq_result* out) {
    API_BEGIN
    NEED(gbm); NEED(european); NEED(cfg); NEED(out);
    ensure_ready();
    run_is(*gbm, *european, z_star, eps, *cfg, *out);
    API_END
}

// ------------------------------------------------------------------ hot-path passes

static PassArgs qmc_args(const mcq_model* m, const mcq_payoff* p, int n_steps, int noise_mode,
                         mcq_handle bb, mcq_handle pca, uint32_t salt_base, int R, uint32_t offset,
                         int64_t n_points, int flags) {
    NEED(m); NEED(p);
    MCQ_REQUIRE(n_points >= 0 && R >= 1, MCQ_ERR_INVALID, "bad R / n_points");
    PassArgs a;
    a.m = m; a.p = p; a.n_steps = n_steps; a.gen = GEN_SOBOL; a.noise = noise_mode;
    a.bb = as_handle(bb, MCQ_NOISE_BB); a.pca = as_handle(pca, MCQ_NOISE_PCA);
    a.salt0 = salt_base; a.R = R; a.offset = offset; a.n_points = (uint64_t)n_points; a.flags = flags;
    return a;
}

int mcq_qmc_pass(const mcq_model* m, const mcq_payoff* p, int n_steps, int noise_mode,
                 mcq_handle bb, mcq_handle pca, uint32_t salt_base, int R, uint32_t offset,
                 int64_t n_points, int flags, double* sums_host) {
    API_BEGIN
    NEED(sums_host);
    PassArgs a = qmc_args(m, p, n_steps, noise_mode, bb, pca, salt_base, R, offset, n_points, flags);
    ensure_ready();
    auto s = pass_sync(engine().ws(0), a);
    std::memcpy(sums_host, s.data(), sizeof(double) * s.size());
    API_END
}

int mcq_qmc_pass_device(const mcq_model* m, const mcq_payoff* p, int n_steps, int noise_mode,
                        mcq_handle bb, mcq_handle pca, uint32_t salt_base, int R, uint32_t offset,
                        int64_t n_points, int flags, double* sums_device, void* stream) {
    API_BEGIN
    NEED(sums_device);
    PassArgs a = qmc_args(m, p, n_steps, noise_mode, bb, pca, salt_base, R, offset, n_points, flags);
    ensure_ready();
    Workspace& ws = engine().ws(0);
    cudaStream_t user = (cudaStream_t)stream;
    if (user) {
        // run on the caller's stream: swap it in for this call
        cudaStream_t own = ws.stream;
        ws.stream = user;
        try { pass_async(ws, a, sums_device); } catch (...) { ws.stream = own; throw; }
        ws.stream = own;
        // the workspace's scratch and status word were used on the caller's stream: later work
        // on the workspace (the next pass, the status read of the next synchronous call) waits
        // for this pass
        join_caller_stream(ws, user);
    } else {
        pass_async(ws, a, sums_device);
    }
    API_END
}

int mcq_mc_pass(const mcq_model* m, const mcq_payoff* p, int n_steps, uint32_t seed,
                uint32_t stream_id, int64_t first_path, int64_t n_paths, double* sums_host) {
    API_BEGIN
    NEED(m); NEED(p); NEED(sums_host);
    MCQ_REQUIRE(first_path >= 0 && n_paths >= 0, MCQ_ERR_INVALID, "bad path range");
    PassArgs a;
    a.m = m; a.p = p; a.n_steps = n_steps; a.gen = GEN_PHILOX; a.R = 1;
    a.offset = (uint64_t)first_path; a.n_points = (uint64_t)n_paths; a.seed = seed; a.stream0 = stream_id;
    ensure_ready();
    auto s = pass_sync(engine().ws(0), a);
    std::memcpy(sums_host, s.data(), sizeof(double) * s.size());
    API_END
}

int mcq_level_pass(const mcq_model* m, const mcq_payoff* p, int n_fine, int M, int noise_mode,
                   mcq_handle bb, mcq_handle pca, int use_sobol, uint32_t seed, uint32_t salt_base,
                   int R, uint32_t offset, int64_t n_points, int flags, double* sums_host) {
    API_BEGIN
    NEED(m); NEED(p); NEED(sums_host);
    MCQ_REQUIRE(R >= 1 && n_points >= 0 && n_fine >= 1, MCQ_ERR_INVALID, "bad level pass sizes");
    PassArgs a;
    a.m = m; a.p = p; a.n_steps = n_fine; a.est = EST_COUPLED;
    a.level0 = (M <= 0);
    a.M = (M <= 0) ? 1 : M;
    a.mlmc_h = true;
    a.gen = use_sobol ? GEN_SOBOL : GEN_PHILOX;
    a.noise = noise_mode;
    a.bb = as_handle(bb, MCQ_NOISE_BB); a.pca = as_handle(pca, MCQ_NOISE_PCA);
    a.seed = seed; a.salt0 = salt_base; a.stream0 = salt_base; a.R = R;
    a.offset = offset; a.n_points = (uint64_t)n_points; a.flags = flags;
    ensure_ready();
    auto s = pass_sync(engine().ws(0), a);
    const int ns = nstat_of(EST_COUPLED, m->kind);   // basket records also carry per-asset deltas
    for (int r = 0; r < R; r++) std::memcpy(sums_host + 4 * r, s.data() + (size_t)ns * r, 4 * sizeof(double));
    API_END
}

int mcq_is_pass(const mcq_model* m, const mcq_payoff* p, int n_steps, double z_star_step, int use_sobol,
                uint32_t seed, uint32_t salt_base, int R, uint32_t offset, int64_t n_points, int flags,
                double* sums_host) {
    API_BEGIN
    NEED(m); NEED(p); NEED(sums_host);
    MCQ_REQUIRE(m->kind == MCQ_MODEL_GBM && p->kind == MCQ_PAYOFF_EUROPEAN, MCQ_ERR_UNSUPPORTED,
                "IS pass: GBM with a European call only (kernel_is_gbm)");
    MCQ_REQUIRE(R >= 1 && n_points >= 0 && n_steps >= 1, MCQ_ERR_INVALID, "bad IS pass sizes");
    PassArgs a;
    a.m = m; a.p = p; a.n_steps = n_steps; a.est = EST_IS;
    a.gen = use_sobol ? GEN_SOBOL : GEN_PHILOX;
    a.seed = seed; a.salt0 = salt_base; a.stream0 = salt_base; a.R = R;
    a.offset = offset; a.n_points = (uint64_t)n_points; a.flags = flags;
    a.z_star = (float)z_star_step;
    ensure_ready();
    auto s = pass_sync(engine().ws(0), a);
    std::memcpy(sums_host, s.data(), sizeof(double) * 2 * R);
    API_END
}

int mcq_debug_pass_dump(const mcq_model* m, int n_steps, int noise_mode, mcq_handle bb,
                        int use_sobol, uint32_t seed, uint32_t salt_base, int R, uint32_t offset,
                        int64_t n_points, int flags, float* out_host) {
    API_BEGIN
    NEED(m); NEED(out_host);
    MCQ_REQUIRE(R >= 1 && n_points >= 1 && n_points <= (1 << 20), MCQ_ERR_INVALID, "bad dump sizes");
    mcq_payoff pay;
    std::memset(&pay, 0, sizeof(pay));
    PassArgs a;
    a.m = m; a.p = &pay; a.n_steps = n_steps; a.gen = use_sobol ? GEN_SOBOL : GEN_PHILOX;
    a.noise = noise_mode;
    if (noise_mode == MCQ_NOISE_PCA) a.pca = as_handle(bb, MCQ_NOISE_PCA);
    else a.bb = as_handle(bb, MCQ_NOISE_BB);
    a.seed = seed; a.salt0 = salt_base;
    a.stream0 = salt_base; a.R = R; a.offset = offset; a.n_points = (uint64_t)n_points; a.flags = flags;
    a.dump = true;
    ensure_ready();
    Workspace& ws = engine().ws(0);
    pass_sync(ws, a);
    const size_t cnt = (size_t)R * n_points * (size_t)(n_steps * noise_dim(*m));
    MCQ_CUDA(cudaMemcpy(out_host, ws.dump.p, sizeof(float) * cnt, cudaMemcpyDeviceToHost));
    API_END
}

// ------------------------------------------------------------------ adjoint Greeks

int mcq_adjoint(const mcq_model* m, const mcq_payoff* p, int n_steps, uint32_t salt_base, int R,
                uint32_t offset, int64_t n_points, int flags, mcq_greeks* out, double* node_vega) {
    API_BEGIN
    NEED(m); NEED(p); NEED(out);
    MCQ_REQUIRE(n_points >= 1 && R >= 1, MCQ_ERR_INVALID, "bad R / n_points");
    ensure_ready();
    adjoint_run(*m, *p, n_steps, salt_base, R, offset, (uint64_t)n_points, flags, *out, node_vega);
    API_END
}

int mcq_book_price(const mcq_book_option* opts, int n, const mcq_mlmc_cfg* ml, const mcq_qmc_cfg* qc,
                   int mode, mcq_book_result* out, mcq_book_stats* stats) {
    API_BEGIN
    NEED(opts); NEED(ml); NEED(qc); NEED(out);
    MCQ_REQUIRE(mode == MCQ_BOOK_BATCHED || mode == MCQ_BOOK_PLAIN, MCQ_ERR_INVALID, "book: unknown mode");
    book_validate(opts, n, *ml, *qc);
    ensure_ready();
    book_price(opts, n, *ml, *qc, mode, out, stats);
    API_END
}

// Book object: owned copies of the submitted options and their arrays.
struct mcq_book_s {
    struct Owned {
        mcq_book_option o;
        std::vector<double> S0, sigma, weights, L;
        mcq_model model{};       // a single-asset option's model and payoff (no arrays: GBM,
        mcq_payoff payoff{};     // Heston, parametric Dupire)
    };
    std::vector<Owned> items;
};

int mcq_book_create(mcq_book* out) {
    API_BEGIN_NOINIT
    NEED(out);
    *out = new mcq_book_s();
    API_END
}

int mcq_book_submit(mcq_book b, const mcq_book_option* opts, int n) {
    API_BEGIN_NOINIT
    NEED(b); NEED(opts);
    MCQ_REQUIRE(n >= 0, MCQ_ERR_INVALID, "book: n must be >= 0");
    std::vector<mcq_book_s::Owned> add((size_t)n);
    for (int i = 0; i < n; i++) {
        const mcq_book_option& o = opts[i];
        mcq_book_s::Owned& w = add[(size_t)i];
        w.o = o;
        if (o.model) {   // single-asset option: copy its model and payoff
            MCQ_REQUIRE(o.payoff, MCQ_ERR_INVALID, "book option " + std::to_string(i) + ": a model needs a payoff");
            w.model = *o.model;
            w.payoff = *o.payoff;
            w.o.S0 = w.o.sigma = w.o.weights = w.o.L = nullptr;
            continue;
        }
        MCQ_REQUIRE(o.n_assets >= 1 && o.n_assets <= MCQ_BOOK_MAX_ASSETS, MCQ_ERR_UNSUPPORTED,
                    "book option " + std::to_string(i) + ": needs 1..16 assets");
        MCQ_REQUIRE(o.S0 && o.sigma, MCQ_ERR_INVALID, "book option " + std::to_string(i) + ": needs S0 and sigma");
        const int d = o.n_assets;
        w.S0.assign(o.S0, o.S0 + d);
        w.sigma.assign(o.sigma, o.sigma + d);
        if (o.weights) w.weights.assign(o.weights, o.weights + d);
        if (o.L) w.L.assign(o.L, o.L + (size_t)d * d);
    }
    for (auto& w : add) b->items.push_back(std::move(w));
    for (auto& w : b->items) {   // re-point at the owned copies (push_back may have moved them)
        if (w.o.model) {
            w.o.model = &w.model;
            w.o.payoff = &w.payoff;
            continue;
        }
        w.o.S0 = w.S0.data();
        w.o.sigma = w.sigma.data();
        w.o.weights = w.weights.empty() ? nullptr : w.weights.data();
        w.o.L = w.L.empty() ? nullptr : w.L.data();
    }
    API_END
}

int mcq_book_size(mcq_book b, int* n) {
    API_BEGIN_NOINIT
    NEED(b); NEED(n);
    *n = (int)b->items.size();
    API_END
}

int mcq_book_run(mcq_book b, const mcq_mlmc_cfg* ml, const mcq_qmc_cfg* qc, int mode, mcq_book_result* out,
                 mcq_book_stats* stats) {
    API_BEGIN
    NEED(b); NEED(ml); NEED(qc); NEED(out);
    MCQ_REQUIRE(!b->items.empty(), MCQ_ERR_INVALID, "book: nothing submitted");
    MCQ_REQUIRE(mode == MCQ_BOOK_BATCHED || mode == MCQ_BOOK_PLAIN, MCQ_ERR_INVALID, "book: unknown mode");
    std::vector<mcq_book_option> opts;
    opts.reserve(b->items.size());
    for (auto& w : b->items) opts.push_back(w.o);
    book_validate(opts.data(), (int)opts.size(), *ml, *qc);
    ensure_ready();
    book_price(opts.data(), (int)opts.size(), *ml, *qc, mode, out, stats);
    API_END
}

int mcq_book_clear(mcq_book b) {
    API_BEGIN_NOINIT
    NEED(b);
    b->items.clear();
    API_END
}

int mcq_book_free(mcq_book b) {
    API_BEGIN_NOINIT
    delete b;
    API_END
}

int mcq_book_level_sums(const mcq_book_option* opt, const mcq_mlmc_cfg* ml, const mcq_qmc_cfg* qc, int level,
                        uint32_t offset, int64_t n_points, double* sums_host) {
    API_BEGIN
    NEED(opt); NEED(ml); NEED(qc); NEED(sums_host);
    book_validate(opt, 1, *ml, *qc);
    MCQ_REQUIRE(level >= 0 && level <= opt->max_L, MCQ_ERR_INVALID, "book: level beyond the option's max_L");
    MCQ_REQUIRE(n_points >= 1 && (uint64_t)offset + (uint64_t)n_points <= (1ull << 32), MCQ_ERR_RANGE,
                "book: n_points >= 1 and offset + n_points <= 2^32");
    ensure_ready();
    book_level_sums(*opt, *ml, *qc, level, offset, n_points, sums_host);
    API_END
}

// ------------------------------------------------------------------ parity exports

static void sobol_export(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n, int flags,
                         int as_normal, void* out_host) {
    MCQ_REQUIRE(dim0 >= 0 && nd >= 1 && dim0 + nd <= 20000, MCQ_ERR_RANGE, "dimensions beyond the Sobol table");
    MCQ_REQUIRE(n >= 0 && (uint64_t)offset + (uint64_t)n <= (1ull << 32), MCQ_ERR_RANGE, "point index beyond 2^32");
    if (n == 0) return;
    ensure_ready();
    Workspace& ws = engine().ws(0);
    const int D = dim0 + nd;
    uint32_t* tab = (uint32_t*)ws.dirs.ensure(sizeof(uint32_t) * 33 * (size_t)D);
    launch_prescramble(engine().d_dv, salt, 1, D, tab, ws.stream);
    ws.dirs_R = -1;   // table no longer matches any cached pass layout
    const size_t bytes = sizeof(uint32_t) * (size_t)nd * (size_t)n;
    void* d = ws.dump.ensure(bytes);
    const float cap = (flags & MCQ_FLAG_COMPAT_U_INF) ? 1.0f : 0x1.fffffep-1f;
    launch_sobol_export(tab, D, dim0, nd, offset, n, cap, as_normal, d, ws.stream);
    MCQ_CUDA(cudaGetLastError());
    MCQ_CUDA(cudaStreamSynchronize(ws.stream));
    MCQ_CUDA(cudaMemcpy(out_host, d, bytes, cudaMemcpyDeviceToHost));
}

int mcq_sobol_hh_u32(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n, uint32_t* out_host) {
    API_BEGIN
    NEED(out_host);
    sobol_export(salt, dim0, nd, offset, n, 0, 0, out_host);
    API_END
}

int mcq_sobol_hh_normal(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n, int flags,
                        float* out_host) {
    API_BEGIN
    NEED(out_host);
    sobol_export(salt, dim0, nd, offset, n, flags, 1, out_host);
    API_END
}

int mcq_debug_wait_timeout(uint32_t polls) {
    API_BEGIN
    MCQ_REQUIRE(polls >= 1 && polls <= (1u << 20), MCQ_ERR_INVALID, "polls must be 1 .. 2^20");
    ensure_ready();
    Workspace& ws = engine().ws(0);
    int* err = arm_err_word(ws);
    launch_wait_probe(err, polls, ws.stream);
    MCQ_CUDA(cudaGetLastError());
    MCQ_CUDA(cudaStreamSynchronize(ws.stream));
    check_err_word(ws);
    API_END
}

int mcq_debug_last_pass_layout(int* groups_per_item, int* carry_words) {
    API_BEGIN
    MCQ_REQUIRE(groups_per_item && carry_words, MCQ_ERR_INVALID, "NULL argument");
    Engine& E = engine();
    *groups_per_item = E.last_gpi;
    *carry_words = E.last_carry;
    API_END
}

int mcq_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    if (!ctr || !key || !out) { g_last_error = "NULL argument"; return MCQ_ERR_INVALID; }
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1; c3 = (uint32_t)p0; c0 = n0; c2 = n2;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
    return MCQ_OK;
}

}  // extern "C"
