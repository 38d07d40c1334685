// drivers.cpp — the adaptive estimators (MC, RQMC, MLMC, MLQMC, control variates, importance
// sampling) as host C++ over the fused pass.  The arithmetic of every driver follows the
// reference's driver line by line (cited per function); what changes is underneath: one fused
// launch per batch / doubling / level round instead of generate -> transform -> price passes
// over D x N arrays, no per-batch allocation, and per-replica sums kept on the device.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <vector>

#include "drivers.h"

namespace mcq {

using Clock = std::chrono::steady_clock;
static double since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

static long long pow2_floor(long long x) {   // methods_cuda.cu:251-255
    long long p = 1;
    while (p * 2 <= x) p *= 2;
    return p;
}

static void check_model_payoff(const mcq_model& m, const mcq_payoff& p) {
    MCQ_REQUIRE(m.kind >= 0 && m.kind <= MCQ_MODEL_BASKET_GBM, MCQ_ERR_INVALID, "unknown model kind");
    MCQ_REQUIRE(p.kind >= 0 && p.kind <= MCQ_PAYOFF_BARRIER_DOWN_OUT, MCQ_ERR_INVALID, "unknown payoff kind");
    MCQ_REQUIRE(m.T > 0, MCQ_ERR_INVALID, "model T must be positive");
}

// ------------------------------------------------------------------ plain MC

// run_mc_fixed_impl (methods_cuda.cu:1173-1265): mean and variance of the mean of n paths.
// Pseudo-random stream: Philox key `seed`, stream id `stream`.
static std::pair<double, double> mc_fixed(Workspace& ws, const mcq_model& m, const mcq_payoff& p,
                                          int n_steps, long long n, uint32_t seed, uint32_t stream,
                                          double* path_steps) {
    PassArgs a;
    a.m = &m; a.p = &p; a.n_steps = n_steps; a.gen = GEN_PHILOX; a.R = 1;
    a.offset = 0; a.n_points = (uint64_t)n; a.seed = seed; a.stream0 = stream;
    std::vector<double> s = pass_sync(ws, a);
    if (path_steps) *path_steps += (double)n * n_steps;
    const double mean = s[0] / n;
    const double var = std::max(0.0, s[1] / n - mean * mean) / n;
    return {mean, var};
}

void run_mc(const mcq_model& m, const mcq_payoff& p, double eps, int n_steps,
            const mcq_mc_cfg& cfg, mcq_result& out) {
    check_model_payoff(m, p);
    MCQ_REQUIRE(eps > 0 && n_steps >= 1 && cfg.pilot_n >= 1, MCQ_ERR_INVALID, "run_mc: bad eps / n_steps / pilot_n");
    auto t0 = Clock::now();
    Workspace& ws = engine().ws(0);
    const int l0 = engine().launches;
    double ps = 0;
    // methods_cuda.cu:1276-1281: pilot, N = 2 Var / eps^2 (at least pilot_n)
    auto [mu_p, var_p] = mc_fixed(ws, m, p, n_steps, cfg.pilot_n, cfg.seed, 0, &ps);
    (void)mu_p;
    const double sample_var = var_p * cfg.pilot_n;
    long long N = (long long)std::ceil(2.0 * sample_var / (eps * eps));
    N = std::max(N, (long long)cfg.pilot_n);
    // :1286-1292 ran the main sample in N_batch batches with seeds seed+1, seed+2, ...; here
    // it is one pass over paths 0..N-1 of an independent stream (id 1).
    PassArgs a;
    a.m = &m; a.p = &p; a.n_steps = n_steps; a.gen = GEN_PHILOX; a.R = 1;
    a.offset = 0; a.n_points = (uint64_t)N; a.seed = cfg.seed; a.stream0 = 1;
    std::vector<double> s = pass_sync(ws, a);
    ps += (double)N * n_steps;
    const double mean = s[0] / N;
    const double var = std::max(0.0, s[1] / N - mean * mean) / N;
    out.price = mean;
    out.std_error = std::sqrt(var);
    out.n_samples = N;
    out.time_s = since(t0);
    out.path_steps = ps;
    out.levels = 1;
    out.launches = engine().launches - l0;
    out.converged = 1;
}

void run_mc_fixed(const mcq_model& m, const mcq_payoff& p, int n_steps, long long n_paths,
                  uint32_t seed, double& mean, double& var_of_mean) {
    check_model_payoff(m, p);
    MCQ_REQUIRE(n_steps >= 1 && n_paths >= 1, MCQ_ERR_INVALID, "run_mc_fixed: bad sizes");
    auto r = mc_fixed(engine().ws(0), m, p, n_steps, n_paths, seed, 0, nullptr);
    mean = r.first;
    var_of_mean = r.second;
}

// ------------------------------------------------------------------ RQMC

// The reference's first points-per-replica (methods_cuda.cu:1521-1533): as many as fit in a
// third of 80 % of free device memory per D floats, capped at INT_MAX/2/D, power of two.
static long long ref_qmc_start(int D, bool use_sobol) {
    long long budget = gpu_free_bytes_80() / 3 / (long long)sizeof(float);
    long long cap = std::max(256LL, budget / std::max(D, 1));
    cap = std::min(cap, (long long)INT_MAX / 2 / std::max(D, 1));
    cap = (cap + 1) & ~1LL;
    long long N = std::max(64LL, cap);
    return use_sobol ? pow2_floor(N) : N;
}

void run_qmc(const mcq_model& m, const mcq_payoff& p, double eps, int n_steps,
             const mcq_qmc_cfg& cfg, int noise, const Handle* bb, const Handle* pca,
             mcq_result& out) {
    check_model_payoff(m, p);
    MCQ_REQUIRE(eps > 0 && n_steps >= 1 && cfg.R >= 1 && cfg.max_doublings >= 1, MCQ_ERR_INVALID,
                "run_qmc: bad eps / n_steps / R / max_doublings");
    auto t0 = Clock::now();
    const int l0 = engine().launches;
    const int D = n_steps * noise_dim(m);
    const bool use_sobol = D <= 20000;
    // the reference falls through to the raw path when the transform handle is missing (:1579-1601)
    if (noise == MCQ_NOISE_BB && !bb) noise = MCQ_NOISE_RAW;
    if (noise == MCQ_NOISE_PCA && !pca) noise = MCQ_NOISE_RAW;
    MCQ_REQUIRE(noise == MCQ_NOISE_RAW || noise_dim(m) == 1, MCQ_ERR_UNSUPPORTED,
                "run_qmc: Brownian bridge / PCA need a one-factor model");
    const int R = cfg.R;
    long long Nper = cfg.N0_per_replica > 0 ? cfg.N0_per_replica : ref_qmc_start(D, use_sobol);
    Workspace& ws = engine().ws(0);
    std::vector<double> acc((size_t)R * 2, 0.0);
    long long Ndone = 0;
    double vom = 1e30, gm = 0.0, ps = 0.0;
    long long total = 0;
    PassArgs a;
    a.m = &m; a.p = &p; a.n_steps = n_steps; a.R = R; a.flags = cfg.flags;
    a.gen = use_sobol ? GEN_SOBOL : GEN_PHILOX;
    a.noise = use_sobol ? noise : MCQ_NOISE_RAW;
    a.bb = bb; a.pca = pca;
    a.salt0 = cfg.salt_base; a.seed = cfg.salt_base; a.stream0 = cfg.salt_base;
    // doubling loop, methods_cuda.cu:1624-1668 (the reference's speculative extra doubling
    // changes only when work is done, not the result)
    for (int dbl = 0; dbl < cfg.max_doublings; dbl++) {
        MCQ_REQUIRE(!use_sobol || (unsigned long long)Nper <= 0xFFFFFFFFull, MCQ_ERR_RANGE,
                    "run_qmc: N_per_replica=" + std::to_string(Nper) + " exceeds the 32-bit Sobol offset");
        if (Nper > Ndone) {
            a.offset = (uint64_t)Ndone;
            a.n_points = (uint64_t)(Nper - Ndone);
            std::vector<double> s = pass_sync(ws, a);
            for (size_t i = 0; i < acc.size(); i++) acc[i] += s[i];
            ps += (double)R * (double)(Nper - Ndone) * n_steps;
            Ndone = Nper;
        }
        double mm = 0.0;
        for (int r = 0; r < R; r++) mm += acc[2 * r] / (double)Nper;
        mm /= R;
        double v = 0.0;
        for (int r = 0; r < R; r++) {
            const double q = acc[2 * r] / (double)Nper - mm;
            v += q * q;
        }
        v = (R > 1) ? v / (R - 1) : 0.0;
        vom = v / R;
        gm = mm;
        total = (long long)R * Nper;
        if (vom < eps * eps / 2.0) break;
        Nper *= 2;
    }
    out.price = gm;
    out.std_error = std::sqrt(vom);
    out.n_samples = total;
    out.time_s = since(t0);
    out.path_steps = ps;
    out.levels = 1;
    out.launches = engine().launches - l0;
    out.converged = (vom < eps * eps / 2.0) ? 1 : 0;
}

// ------------------------------------------------------------------ MLMC

void run_mlmc(const mcq_model& m, const mcq_payoff& p, double eps, const mcq_mlmc_cfg& cfg,
              mcq_result& out) {
    check_model_payoff(m, p);
    // the reference refuses baskets here (methods_cuda.cu:1318-1320); the engine couples the
    // correlated GBM and Dupire baskets of up to kMaxBasket assets (BasketLevelC)
    MCQ_REQUIRE((m.kind != MCQ_MODEL_MULTI_DUPIRE && m.kind != MCQ_MODEL_BASKET_GBM) || m.n_assets <= kMaxBasket,
                MCQ_ERR_UNSUPPORTED, "run_mlmc: coupled baskets take at most 16 assets");
    MCQ_REQUIRE(eps > 0 && cfg.M >= 2 && cfg.max_L >= 2 && cfg.pilot_n >= 1 && cfg.n0_steps >= 1,
                MCQ_ERR_INVALID, "run_mlmc: bad eps / M / max_L / pilot_n / n0_steps");
    auto t0 = Clock::now();
    const int l0c = engine().launches;
    const int M = cfg.M, max_L = cfg.max_L;
    int L = 2;
    std::vector<double> E(max_L + 1, 0.0), V(max_L + 1, 0.0);
    std::vector<long long> N(max_L + 1, 0);
    std::vector<double*> dsum(max_L + 1, nullptr);
    double ps = 0.0;
    uint32_t seed_ctr = 0;   // one fresh Philox stream per launch (the reference: seed 42, 43, ...)

    auto nfine = [&](int l) -> long long {
        long long n = cfg.n0_steps;
        for (int i = 0; i < l; i++) n *= M;
        return n;
    };
    // launch_level (methods_cuda.cu:1347-1395), asynchronous on the level's own stream
    auto launch = [&](int l, long long n) {
        Workspace& w = engine().ws(1 + l);
        const long long nf = nfine(l);
        MCQ_REQUIRE(nf <= INT_MAX / 4, MCQ_ERR_RANGE, "run_mlmc: level step count overflow");
        PassArgs a;
        a.m = &m; a.p = &p; a.n_steps = (int)nf; a.est = EST_COUPLED; a.M = M; a.level0 = (l == 0);
        a.mlmc_h = true; a.gen = GEN_PHILOX; a.R = 1; a.offset = 0; a.n_points = (uint64_t)n;
        a.seed = cfg.seed; a.stream0 = seed_ctr++; a.flags = cfg.flags;
        dsum[l] = (double*)w.sums.ensure((size_t)nstat_of(EST_COUPLED, m.kind) * sizeof(double));
        pass_async(w, a, dsum[l]);
        ps += (double)n * (double)(nf + (l ? nf / M : 0));
    };
    // collect_level (:1400-1409)
    auto collect = [&](int l) -> std::vector<double> {
        Workspace& w = engine().ws(1 + l);
        double* h = (double*)w.hsums.ensure(4 * sizeof(double));
        MCQ_CUDA(cudaMemcpyAsync(h, dsum[l], 4 * sizeof(double), cudaMemcpyDeviceToHost, w.stream));   // first 4 stats
        MCQ_CUDA(cudaStreamSynchronize(w.stream));
        check_err_word(w);
        return std::vector<double>(h, h + 4);
    };

    for (int l = 0; l <= L; l++) launch(l, cfg.pilot_n);   // :1412-1421
    for (int l = 0; l <= L; l++) {
        auto s = collect(l);
        const long long np = cfg.pilot_n;
        const double em = s[0] / np;
        V[l] = std::max(0.0, s[1] / np - em * em);
        E[l] = em;
        N[l] = np;
    }
    bool converged = false;
    int iter = 0;
    while (!converged && L <= max_L && iter++ < 50) {   // :1426-1473
        double sum_term = 0.0;
        for (int l = 0; l <= L; l++) sum_term += std::sqrt(V[l] * std::pow((double)M, l));
        std::vector<long long> extra(L + 1, 0);
        for (int l = 0; l <= L; l++) {
            const double Cl = std::pow((double)M, l);
            long long Nopt = (long long)std::ceil(2.0 / (eps * eps) * std::sqrt(V[l] / Cl) * sum_term);
            Nopt = std::max(Nopt, 100LL);
            if (Nopt > N[l]) {
                extra[l] = Nopt - N[l];
                launch(l, extra[l]);
            }
        }
        for (int l = 0; l <= L; l++) {
            if (extra[l] > 0) {
                auto s = collect(l);
                const long long Nn = N[l] + extra[l];
                const double tsum = E[l] * N[l] + s[0];
                const double ts2 = (V[l] + E[l] * E[l]) * N[l] + s[1];
                E[l] = tsum / Nn;
                V[l] = std::max(0.0, ts2 / Nn - E[l] * E[l]);
                N[l] = Nn;
            }
        }
        double bias = std::abs(E[L]) / (M - 1);
        if (L >= 1) bias = std::max(bias, std::abs(E[L - 1]) * M / (double)(M * M - M));
        converged = bias < eps / std::sqrt(2.0);
        if (!converged && L < max_L) {
            L++;
            launch(L, cfg.pilot_n);
            auto s = collect(L);
            const long long np = cfg.pilot_n;
            const double em = s[0] / np;
            V[L] = std::max(0.0, s[1] / np - em * em);
            E[L] = em;
            N[L] = np;
        }
    }
    double price = 0.0, vs = 0.0;
    long long Nt = 0;
    for (int l = 0; l <= L; l++) {   // :1478-1486
        price += E[l];
        vs += N[l] > 0 ? V[l] / N[l] : 0.0;
        Nt += N[l];
    }
    out.price = price;
    out.std_error = std::sqrt(vs);
    out.n_samples = Nt;
    out.time_s = since(t0);
    out.path_steps = ps;
    out.levels = L + 1;
    out.launches = engine().launches - l0c;
    out.converged = converged ? 1 : 0;
}

// ------------------------------------------------------------------ MLQMC

void run_mlqmc(const mcq_model& m, const mcq_payoff& p, double eps, const mcq_mlmc_cfg& ml,
               const mcq_qmc_cfg& qc, int noise, const std::vector<const Handle*>& bb_list,
               const std::vector<const Handle*>& pca_list, mcq_result& out) {
    check_model_payoff(m, p);
    // the reference refuses baskets here (methods_cuda.cu:1695-1697); the engine couples the
    // correlated GBM and Dupire baskets of up to kMaxBasket assets (BasketLevelC)
    MCQ_REQUIRE((m.kind != MCQ_MODEL_MULTI_DUPIRE && m.kind != MCQ_MODEL_BASKET_GBM) || m.n_assets <= kMaxBasket,
                MCQ_ERR_UNSUPPORTED, "run_mlqmc: coupled baskets take at most 16 assets");
    MCQ_REQUIRE(noise == MCQ_NOISE_RAW || noise_dim(m) == 1, MCQ_ERR_UNSUPPORTED,
                "run_mlqmc: Brownian bridge / PCA only for one-factor models (:1702-1704)");
    MCQ_REQUIRE(eps > 0 && ml.M >= 2 && ml.max_L >= 2 && ml.pilot_n >= 1 && ml.n0_steps >= 1 && qc.R >= 1,
                MCQ_ERR_INVALID, "run_mlqmc: bad eps / M / max_L / pilot_n / n0_steps / R");
    auto t0 = Clock::now();
    const int l0c = engine().launches;
    const int M = ml.M, max_L = ml.max_L, R = qc.R;
    const int ns = nstat_of(EST_COUPLED, m.kind);   // record stride per replica
    int L = 2;
    std::vector<double> E(max_L + 1, 0.0), sig2(max_L + 1, 0.0);
    std::vector<long long> N(max_L + 1, 0), next_off(max_L + 1, 0);
    std::vector<double*> dsum(max_L + 1, nullptr);
    double ps = 0.0;
    auto nfine = [&](int l) -> long long {
        long long n = ml.n0_steps;
        for (int i = 0; i < l; i++) n *= M;
        return n;
    };
    // launch_level (methods_cuda.cu:1793-1922): all R replicas of the level in one pass,
    // salts salt_base + l R + r, shared offset next_off[l]
    auto launch = [&](int l, long long n) {
        Workspace& w = engine().ws(1 + l);
        const long long nf = nfine(l);
        MCQ_REQUIRE(nf <= INT_MAX / 4, MCQ_ERR_RANGE, "run_mlqmc: level step count overflow");
        const long long D = nf * noise_dim(m);
        const bool use_sobol = D <= 20000;
        const Handle* bbh = nullptr;
        if (noise == MCQ_NOISE_BB) {
            MCQ_REQUIRE(l < (int)bb_list.size() && bb_list[l], MCQ_ERR_INVALID,
                        "run_mlqmc: missing bb_list[" + std::to_string(l) + "]");
            MCQ_REQUIRE(bb_list[l]->n == nf, MCQ_ERR_INVALID,
                        "run_mlqmc: bb_list[" + std::to_string(l) + "] has N=" + std::to_string(bb_list[l]->n) +
                            ", expected " + std::to_string(nf));
            bbh = bb_list[l];
        }
        if (noise == MCQ_NOISE_PCA) {
            MCQ_REQUIRE(l < (int)pca_list.size() && pca_list[l], MCQ_ERR_INVALID,
                        "run_mlqmc: missing pca_list[" + std::to_string(l) + "]");
            MCQ_REQUIRE(pca_list[l]->n == nf, MCQ_ERR_INVALID, "run_mlqmc: pca_list size mismatch");
        }
        MCQ_REQUIRE(!use_sobol || (unsigned long long)(next_off[l] + n) <= 0xFFFFFFFFull, MCQ_ERR_RANGE,
                    "run_mlqmc: level " + std::to_string(l) + " offset exceeds the 32-bit Sobol limit");
        PassArgs a;
        a.m = &m; a.p = &p; a.n_steps = (int)nf; a.est = EST_COUPLED; a.M = M; a.level0 = (l == 0);
        a.mlmc_h = true; a.R = R; a.flags = ml.flags | qc.flags;
        a.gen = use_sobol ? GEN_SOBOL : GEN_PHILOX;
        a.noise = use_sobol ? noise : MCQ_NOISE_RAW;
        a.bb = bbh;
        a.pca = (noise == MCQ_NOISE_PCA && l < (int)pca_list.size()) ? pca_list[l] : nullptr;
        a.salt0 = qc.salt_base + (uint32_t)(l * R);
        a.seed = qc.salt_base; a.stream0 = qc.salt_base + (uint32_t)(l * R);
        a.offset = (uint64_t)next_off[l];
        a.n_points = (uint64_t)n;
        dsum[l] = (double*)w.sums.ensure((size_t)R * ns * sizeof(double));
        pass_async(w, a, dsum[l]);
        next_off[l] += n;
        ps += (double)R * (double)n * (double)(nf + (l ? nf / M : 0));
    };
    // collect_level (:1927-1944): mean and sample variance of the R replica means
    auto collect = [&](int l, long long n) -> std::pair<double, double> {
        Workspace& w = engine().ws(1 + l);
        double* h = (double*)w.hsums.ensure((size_t)R * ns * sizeof(double));
        MCQ_CUDA(cudaMemcpyAsync(h, dsum[l], (size_t)R * ns * sizeof(double), cudaMemcpyDeviceToHost, w.stream));
        MCQ_CUDA(cudaStreamSynchronize(w.stream));
        check_err_word(w);
        double mm = 0.0;
        for (int r = 0; r < R; r++) mm += h[ns * r] / n;
        mm /= R;
        double v = 0.0;
        for (int r = 0; r < R; r++) {
            const double q = h[ns * r] / n - mm;
            v += q * q;
        }
        v = (R > 1) ? v / (R - 1) : 0.0;
        return {mm, v};
    };
    const long long Np = ml.pilot_n;
    for (int l = 0; l <= L; l++) launch(l, Np);
    for (int l = 0; l <= L; l++) {
        auto [em, vv] = collect(l, Np);
        E[l] = em; sig2[l] = vv * (double)Np; N[l] = Np;
    }
    bool converged = false;
    int iter = 0;
    while (!converged && L <= max_L && iter++ < 50) {   // :1950-2000
        double sum_term = 0.0;
        for (int l = 0; l <= L; l++) sum_term += std::sqrt(sig2[l] * std::pow((double)M, l));
        std::vector<long long> extra(L + 1, 0);
        for (int l = 0; l <= L; l++) {
            const double Cl = std::pow((double)M, l);
            long long Nopt = (long long)std::ceil(2.0 / ((double)R * eps * eps) * std::sqrt(sig2[l] / Cl) * sum_term);
            Nopt = std::max(Nopt, 100LL);
            if (Nopt > N[l]) {
                extra[l] = Nopt - N[l];
                launch(l, extra[l]);
            }
        }
        for (int l = 0; l <= L; l++) {
            if (extra[l] > 0) {
                auto [em, vv] = collect(l, extra[l]);
                const double wo = (double)N[l], wn = (double)extra[l];
                const double s2n = vv * wn;
                E[l] = (E[l] * wo + em * wn) / (wo + wn);
                sig2[l] = (sig2[l] * wo + s2n * wn) / (wo + wn);
                N[l] += extra[l];
            }
        }
        double bias = std::abs(E[L]) / std::max(M - 1, 1);
        if (L >= 1) bias = std::max(bias, std::abs(E[L - 1]) * M / (double)std::max(M * (M - 1), 1));
        converged = bias < eps / std::sqrt(2.0);
        if (!converged && L < max_L) {
            L++;
            launch(L, Np);
            auto [em, vv] = collect(L, Np);
            E[L] = em; sig2[L] = vv * (double)Np; N[L] = Np;
        }
    }
    double price = 0.0, vs = 0.0;
    long long Nt = 0;
    for (int l = 0; l <= L; l++) {   // :2010-2016
        price += E[l];
        vs += sig2[l] / ((double)N[l] * (double)R);
        Nt += N[l] * R;
    }
    out.price = price;
    out.std_error = std::sqrt(vs);
    out.n_samples = Nt;
    out.time_s = since(t0);
    out.path_steps = ps;
    out.levels = L + 1;
    out.launches = engine().launches - l0c;
    out.converged = converged ? 1 : 0;
}

// ------------------------------------------------------------------ control variates

static int cv_est(const mcq_model& main_m) {
    if (main_m.kind == MCQ_MODEL_GBM) return EST_CV_ASIAN;        // kernel_gbm_asian_cv
    if (main_m.kind == MCQ_MODEL_DUPIRE) return EST_CV_DUPIRE;    // kernel_dupire_gbm_cv
    throw Error(MCQ_ERR_UNSUPPORTED, "control variates: main model must be GBM (Asian/geometric) or Dupire (GBM control)");
}

// cv_pilot (methods_cuda.cu:2026-2076)
void cv_pilot(const mcq_model& main_m, const mcq_payoff& main_p, double E_ctrl, int n_steps,
              int N_pilot, uint32_t seed, mcq_cv_pilot_out& out) {
    MCQ_REQUIRE(n_steps >= 1 && N_pilot >= 2, MCQ_ERR_INVALID, "cv_pilot: bad sizes");
    PassArgs a;
    a.m = &main_m; a.p = &main_p; a.n_steps = n_steps; a.est = cv_est(main_m); a.gen = GEN_PHILOX;
    a.R = 1; a.offset = 0; a.n_points = (uint64_t)N_pilot; a.seed = seed; a.stream0 = 0;
    a.beta_cv = 0.0f; a.E_ctrl = (float)E_ctrl;
    auto hs = pass_sync(engine().ws(0), a);
    const double Nd = (double)N_pilot;
    const double Ea = hs[0] / Nd, Ea2 = hs[1] / Nd, Eg = hs[4] / Nd, Eg2 = hs[5] / Nd, Eag = hs[6] / Nd;
    const double vmain = std::max(0.0, Ea2 - Ea * Ea);
    const double vctrl = std::max(1e-30, Eg2 - Eg * Eg);
    const double cov = Eag - Ea * Eg;
    out.beta = std::clamp(cov / vctrl, 0.0, 5.0);
    out.var_plain = vmain;
    out.var_cv = std::max(0.0, vmain - cov * cov / vctrl);
}

// run_mc_cv_cuda (methods_cuda.cu:2078-2163)
void run_mc_cv(const mcq_model& main_m, const mcq_payoff& main_p, double E_ctrl, double beta,
               double eps, int n_steps, const mcq_mc_cfg& cfg, mcq_result& out) {
    MCQ_REQUIRE(eps > 0 && n_steps >= 1 && cfg.pilot_n >= 2, MCQ_ERR_INVALID, "run_mc_cv: bad arguments");
    auto t0 = Clock::now();
    const int l0c = engine().launches;
    Workspace& ws = engine().ws(0);
    PassArgs a;
    a.m = &main_m; a.p = &main_p; a.n_steps = n_steps; a.est = cv_est(main_m); a.gen = GEN_PHILOX;
    a.R = 1; a.offset = 0; a.n_points = (uint64_t)cfg.pilot_n; a.seed = cfg.seed; a.stream0 = 0;
    a.beta_cv = (float)beta; a.E_ctrl = (float)E_ctrl;
    auto hs = pass_sync(ws, a);
    const double mu_cv = hs[2] / cfg.pilot_n;
    const double var_cv = std::max(0.0, hs[3] / cfg.pilot_n - mu_cv * mu_cv);
    long long N = (long long)std::ceil(2.0 * var_cv / (eps * eps));
    N = std::max(N, (long long)cfg.pilot_n);
    N = (N + 1) & ~1LL;   // the reference's even count (:2131), kept so N matches
    a.n_points = (uint64_t)N;
    a.stream0 = 100;      // the reference's main run uses seed + 100 (:2144)
    hs = pass_sync(ws, a);
    const double mean = hs[2] / N;
    const double var = std::max(0.0, hs[3] / N - mean * mean) / N;
    out.price = mean;
    out.std_error = std::sqrt(var);
    out.n_samples = N;
    out.time_s = since(t0);
    out.path_steps = (double)(cfg.pilot_n + N) * n_steps;
    out.levels = 1;
    out.launches = engine().launches - l0c;
    out.converged = 1;
}

// run_qmc_cv_cuda (methods_cuda.cu:2165-2278)
void run_qmc_cv(const mcq_model& main_m, const mcq_payoff& main_p, double E_ctrl, double beta,
                double eps, int n_steps, const mcq_qmc_cfg& cfg, mcq_result& out) {
    MCQ_REQUIRE(eps > 0 && n_steps >= 1 && cfg.R >= 1 && cfg.max_doublings >= 1, MCQ_ERR_INVALID,
                "run_qmc_cv: bad arguments");
    auto t0 = Clock::now();
    const int l0c = engine().launches;
    Workspace& ws = engine().ws(0);
    const int R = cfg.R;
    long long Nper;
    if (cfg.N0_per_replica > 0) {
        Nper = cfg.N0_per_replica;
    } else {   // :2188-2190
        long long budget = gpu_free_bytes_80() / (long long)sizeof(float);
        Nper = pow2_floor(std::max(512LL, budget / std::max(n_steps, 1)));
    }
    PassArgs a;
    a.m = &main_m; a.p = &main_p; a.n_steps = n_steps; a.est = cv_est(main_m); a.gen = GEN_SOBOL;
    a.R = R; a.salt0 = cfg.salt_base; a.flags = cfg.flags;
    a.beta_cv = (float)beta; a.E_ctrl = (float)E_ctrl;
    MCQ_REQUIRE(n_steps <= 20000, MCQ_ERR_RANGE, "run_qmc_cv: dimension beyond the Sobol table");
    std::vector<double> acc((size_t)R * 7, 0.0);
    long long Ndone = 0;
    double vom = 1e30, gm = 0.0, ps = 0.0;
    long long total = 0;
    for (int dbl = 0; dbl < cfg.max_doublings; dbl++) {
        MCQ_REQUIRE((unsigned long long)Nper <= 0xFFFFFFFFull, MCQ_ERR_RANGE,
                    "run_qmc_cv: N_per_rep exceeds the 32-bit Sobol offset");
        if (Nper > Ndone) {
            a.offset = (uint64_t)Ndone;
            a.n_points = (uint64_t)(Nper - Ndone);
            auto s = pass_sync(ws, a);
            for (size_t i = 0; i < acc.size(); i++) acc[i] += s[i];
            ps += (double)R * (double)(Nper - Ndone) * n_steps;
            Ndone = Nper;
        }
        double mm = 0.0;
        for (int r = 0; r < R; r++) mm += acc[7 * r + 2] / (double)Nper;
        mm /= R;
        double v = 0.0;
        for (int r = 0; r < R; r++) {
            const double q = acc[7 * r + 2] / (double)Nper - mm;
            v += q * q;
        }
        v = (R > 1) ? v / (R - 1) : 0.0;
        vom = v / R;
        gm = mm;
        total = (long long)R * Nper;
        if (vom < eps * eps / 2.0) break;
        Nper *= 2;
    }
    out.price = gm;
    out.std_error = std::sqrt(vom);
    out.n_samples = total;
    out.time_s = since(t0);
    out.path_steps = ps;
    out.levels = 1;
    out.launches = engine().launches - l0c;
    out.converged = 1;
}

// ------------------------------------------------------------------ importance sampling

// run_is_cuda (methods_cuda.cu:2285-2365)
void run_is(const mcq_model& gbm, const mcq_payoff& eur, double z_star, double eps,
            const mcq_mc_cfg& cfg, mcq_result& out) {
    MCQ_REQUIRE(gbm.kind == MCQ_MODEL_GBM && eur.kind == MCQ_PAYOFF_EUROPEAN, MCQ_ERR_UNSUPPORTED,
                "run_is: GBM with a European call only");
    MCQ_REQUIRE(eps > 0 && cfg.pilot_n >= 2, MCQ_ERR_INVALID, "run_is: bad arguments");
    auto t0 = Clock::now();
    const int l0c = engine().launches;
    Workspace& ws = engine().ws(0);
    const int n_steps = std::max(4, (int)std::ceil(gbm.T / eps));   // :2296
    PassArgs a;
    a.m = &gbm; a.p = &eur; a.n_steps = n_steps; a.est = EST_IS; a.gen = GEN_PHILOX; a.R = 1;
    a.offset = 0; a.n_points = (uint64_t)cfg.pilot_n; a.seed = cfg.seed; a.stream0 = 0;
    a.z_star = (float)(z_star / std::sqrt((double)n_steps));   // :2297
    auto hs = pass_sync(ws, a);
    const double mu = hs[0] / cfg.pilot_n;
    const double var = std::max(0.0, hs[1] / cfg.pilot_n - mu * mu);
    long long N = (long long)std::ceil(2.0 * var / (eps * eps));
    N = std::max(N, (long long)cfg.pilot_n);
    N = (N + 1) & ~1LL;
    a.n_points = (uint64_t)N;
    a.stream0 = 1;   // :2338 seed + 1
    hs = pass_sync(ws, a);
    const double mean = hs[0] / N;
    const double vf = std::max(0.0, hs[1] / N - mean * mean) / N;
    out.price = mean;
    out.std_error = std::sqrt(vf);
    out.n_samples = N;
    out.time_s = since(t0);
    out.path_steps = (double)(cfg.pilot_n + N) * n_steps;
    out.levels = 1;
    out.launches = engine().launches - l0c;
    out.converged = 1;
}

}  // namespace mcq
