// mcq.hpp — the reference's C++ API (methods_cuda.cuh, models.hpp, payoffs.hpp, utils.hpp of
// QuantGuy3/financial-derivatives-montecarlo) re-created over the engine's C ABI (mcq.h).
//
// Callers written against the reference compile unchanged: a `methods_cuda.cuh` that
// includes this header is all they need.  Names, fields, defaults and signatures follow the
// reference so that source stays compatible; every function body is this engine's.  Errors
// that the C ABI reports as status codes are rethrown as std::runtime_error, as the reference
// throws.
#pragma once

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdio>
#include <functional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <variant>
#include <vector>

#include "mcq.h"

// ------------------------------------------------------------------ models (models.hpp)

inline constexpr int CONST_DIM_MAX = 64;
inline constexpr int D_MAX_SOBOL = 20000;

struct GBMParams {
    double S0 = 100.0, mu = 0.05, sigma = 0.20, T = 1.0;
};

struct HestonParams {
    double S0 = 100.0, mu = 0.05, kappa = 2.0, theta = 0.04, xi = 0.5, rho = -0.9, v0 = 0.04, T = 1.0;
    double L[2][2] = {};   // second row drives dW2 = L10 Z1 + L11 Z2, as the reference
    void compute_cholesky() {
        L[0][0] = 1.0; L[0][1] = 0.0;
        L[1][0] = rho; L[1][1] = std::sqrt(1.0 - rho * rho);
    }
};

struct DupireLocalParams {
    double S0 = 100.0, mu = 0.05, sigma0 = 0.20, alpha = 0.5, beta_d = 0.7, T = 1.0;
};

struct MultiDupireParams {
    int n = 100;
    double mu = 0.05, sigma0 = 0.20, alpha = 0.5, beta_d = 0.7, T = 1.0;
    bool uncorrelated = false;
    std::vector<double> S0;
    std::vector<double> L;
};

using ModelVariant = std::variant<GBMParams, HestonParams, DupireLocalParams, MultiDupireParams>;

inline int model_noise_dim(const ModelVariant& mv) {
    return std::visit([](const auto& m) -> int {
        using T = std::decay_t<decltype(m)>;
        if constexpr (std::is_same_v<T, HestonParams>) return 2;
        else if constexpr (std::is_same_v<T, MultiDupireParams>) return m.n;
        else return 1;
    }, mv);
}
inline double model_T(const ModelVariant& mv) {
    return std::visit([](const auto& m) { return m.T; }, mv);
}
inline double model_S0(const ModelVariant& mv) {
    return std::visit([](const auto& m) -> double {
        using T = std::decay_t<decltype(m)>;
        if constexpr (std::is_same_v<T, MultiDupireParams>) return m.S0.empty() ? 100.0 : m.S0[0];
        else return m.S0;
    }, mv);
}

// ------------------------------------------------------------------ payoffs (payoffs.hpp)

inline constexpr double BGK_BETA = 0.5826;
inline constexpr float BGK_BETA_F = 0.5826f;

struct European { double K, r, T; };
struct Asian { double K; };
struct GeomAsian { double K; };
struct Lookback { double sigma; };
struct Barrier { double K, B, sigma, r, T; };
struct Basket { double K, r, T; int n_assets; };

using PayoffVariant = std::variant<European, Asian, GeomAsian, Lookback, Barrier, Basket>;

inline bool payoff_needs_full_path(const PayoffVariant& pv) {
    return std::holds_alternative<Asian>(pv) || std::holds_alternative<GeomAsian>(pv) ||
           std::holds_alternative<Lookback>(pv) || std::holds_alternative<Barrier>(pv);
}
inline double payoff_discount(const PayoffVariant& pv) {
    return std::visit([](const auto& p) -> double {
        using T = std::decay_t<decltype(p)>;
        if constexpr (std::is_same_v<T, European> || std::is_same_v<T, Barrier> || std::is_same_v<T, Basket>)
            return std::exp(-p.r * p.T);
        else return 1.0;
    }, pv);
}

// ------------------------------------------------------------------ host helpers (utils.hpp)

inline double mcq_norm_cdf(double x) { return 0.5 * std::erfc(-x / std::sqrt(2.0)); }

inline double bs_call(double S0, double K, double T, double r, double sigma) {
    if (T <= 0.0 || sigma <= 0.0) return std::max(S0 - K * std::exp(-r * T), 0.0);
    const double sT = std::sqrt(T);
    const double d1 = (std::log(S0 / K) + (r + 0.5 * sigma * sigma) * T) / (sigma * sT), d2 = d1 - sigma * sT;
    return S0 * mcq_norm_cdf(d1) - K * std::exp(-r * T) * mcq_norm_cdf(d2);
}

// Discrete geometric-average call under GBM, undiscounted, average over S_1..S_n.
inline double geom_asian_analytic(double S0, double K, double T, double mu, double sigma, int n) {
    const double m = std::log(S0) + (mu - 0.5 * sigma * sigma) * T * (n + 1) / (2.0 * n);
    const double v = sigma * sigma * T * (n + 1) * (2.0 * n + 1) / (6.0 * n * n), s = std::sqrt(v);
    if (s < 1e-12) return std::max(std::exp(m) - K, 0.0);
    const double d1 = (m + v - std::log(K)) / s;
    return std::exp(m + 0.5 * v) * mcq_norm_cdf(d1) - K * mcq_norm_cdf(d1 - s);
}

struct BBData {
    int N;
    double T;
    std::vector<int> map_idx, left_idx, right_idx;
    std::vector<double> weight_left, weight_right, std_dev;
};

// Dyadic bridge in level order: step 0 fixes W[N]; then the midpoints of each level.
inline BBData bb_precompute(int N, double T) {
    assert(N > 0 && (N & (N - 1)) == 0);
    BBData bb{N, T, std::vector<int>(N, 0), std::vector<int>(N, 0), std::vector<int>(N, 0),
              std::vector<double>(N, 0.0), std::vector<double>(N, 0.0), std::vector<double>(N, 0.0)};
    bb.map_idx[0] = N;
    bb.std_dev[0] = std::sqrt(T);
    int step = 1;
    for (int stride = N; stride > 1; stride >>= 1)
        for (int L = 0; L < N; L += stride) {
            const int R = L + stride, M = L + stride / 2;
            const double tL = L * T / N, tR = R * T / N, tM = M * T / N;
            bb.map_idx[step] = M; bb.left_idx[step] = L; bb.right_idx[step] = R;
            bb.weight_left[step] = (tR - tM) / (tR - tL);
            bb.weight_right[step] = (tM - tL) / (tR - tL);
            bb.std_dev[step] = std::sqrt((tM - tL) * (tR - tM) / (tR - tL));
            step++;
        }
    return bb;
}

inline void bb_apply(const BBData& bb, double* Z, double* dW, int n_sim) {
    std::vector<double> W(bb.N + 1);
    for (int s = 0; s < n_sim; s++) {
        const double* z = Z + (size_t)s * bb.N;
        std::fill(W.begin(), W.end(), 0.0);
        W[bb.map_idx[0]] = bb.std_dev[0] * z[0];
        for (int k = 1; k < bb.N; k++)
            W[bb.map_idx[k]] = bb.weight_left[k] * W[bb.left_idx[k]] + bb.weight_right[k] * W[bb.right_idx[k]] +
                               bb.std_dev[k] * z[k];
        for (int k = 0; k < bb.N; k++) dW[(size_t)s * bb.N + k] = W[k + 1] - W[k];
    }
}

struct PCAData {
    int m;
    double T;
    std::vector<double> M_pca;     // column-major m x m: dW = M_pca z
    std::vector<float> M_pca_f32;
};

// Principal components of the Brownian covariance h min(i+1, j+1): the eigenpairs are known in
// closed form (eigenvalue h / (4 sin^2((2k+1) pi / (2(2m+1))))), sorted descending, signs fixed
// by a positive first component; M_pca is the row difference of V sqrt(Lambda).
inline PCAData pca_compute(int m, double T) {
    PCAData p{m, T, std::vector<double>((size_t)m * m), std::vector<float>((size_t)m * m)};
    const double h = T / m, den = 2.0 * m + 1.0, pi = 3.14159265358979323846;
    for (int k = 0; k < m; k++) {
        const double s = std::sin((2.0 * k + 1.0) * pi / (2.0 * den));
        const double sl = std::sqrt(h / (4.0 * s * s)), c = 2.0 / std::sqrt(den);
        double prev = 0.0;
        for (int i = 0; i < m; i++) {
            const double cum = c * std::sin((2.0 * k + 1.0) * (i + 1.0) * pi / den) * sl;
            p.M_pca[(size_t)k * m + i] = cum - prev;
            prev = cum;
        }
    }
    for (size_t i = 0; i < p.M_pca.size(); i++) p.M_pca_f32[i] = (float)p.M_pca[i];
    return p;
}

using SimFn = std::function<double(int n_steps, long long n_paths, unsigned seed)>;

// Two-level Richardson estimate of the weak-error constant (bias(h) ~ c1 h); returns 1/c1.
inline double estimar_c1_richardson(SimFn sim_fn, double T, int M_rich, int N_pilot, unsigned seed = 0) {
    const int n_fine = std::max(4 * M_rich, 4), n_coarse = n_fine / M_rich;
    const double Pf = sim_fn(n_fine, N_pilot, seed), Pc = sim_fn(n_coarse, N_pilot, seed + 1);
    double c = std::abs(Pc - Pf) / ((T / n_fine) * (M_rich - 1));
    if (c < 1e-12) c = 1e-12;
    return 1.0 / c;
}

struct RunningStats {
    double mean = 0.0, M2 = 0.0;
    long long n = 0;
    void update(double x) {
        ++n;
        const double d = x - mean;
        mean += d / n;
        M2 += d * (x - mean);
    }
    double variance() const { return n > 1 ? M2 / (n - 1) : 0.0; }
    double std_error() const { return n > 0 ? std::sqrt(variance() / n) : 0.0; }
};

struct TableRow {
    std::string method;
    double price, std_error;
    long long n_samples;
    double time_s;
};

// Same layout as the reference's table (parsed by its report scripts).
inline void print_table(const std::vector<TableRow>& rows, double price_ref, double epsilon,
                        const std::string& example_name) {
    std::printf("\n[%s]   epsilon = %g\n", example_name.c_str(), epsilon);
    std::printf("  Referencia: %.6f\n\n", price_ref);
    std::printf("  %-22s%10s%10s%12s%9s%10s%6s\n", "Metodo", "Precio", "StdErr", "N", "T(s)", "|Error|", "OK?");
    std::printf("  %s\n", std::string(79, '-').c_str());
    for (const auto& r : rows) {
        const double err = std::abs(r.price - price_ref);
        std::printf("  %-22s%10.4f%10.4f%12lld%9.3f%10.4f%6s\n", r.method.c_str(), r.price, r.std_error,
                    r.n_samples, r.time_s, err, err < 2.0 * epsilon ? "SI" : "NO");
    }
    std::printf("\n");
}

// ------------------------------------------------------------------ drivers (methods_cuda.cuh)

struct MCConfig {
    long long N_batch = 1LL << 16;
    int pilot_n = 10000;
    unsigned seed = 123u;
};
struct QMCConfig {
    int R = 32;
    int max_doublings = 20;
};
struct MLMCConfig {
    int M = 2;
    int max_L = 10;
    int pilot_n = 400;
};
enum class NoiseMode { Raw, BrownianBridge, PCA };
struct MCResult {
    double price = 0.0, std_error = 0.0;
    long long n_samples = 0;
    double time_s = 0.0;
};
struct CVPilot { double beta, var_plain, var_cv; };

struct DeviceBBData { mcq_handle h = nullptr; int N = 0; };
struct DevicePCAData { mcq_handle h = nullptr; int m = 0; };

namespace mcq_detail {

inline void check(int rc) {
    if (rc != MCQ_OK) throw std::runtime_error(std::string("mcq: ") + mcq_last_error());
}

// mcq_model / mcq_payoff views of the variants; vectors stay owned by the caller's objects.
inline mcq_model to_c(const ModelVariant& mv) {
    mcq_model m{};
    std::visit([&](const auto& x) {
        using T = std::decay_t<decltype(x)>;
        m.T = x.T;
        if constexpr (std::is_same_v<T, GBMParams>) {
            m.kind = MCQ_MODEL_GBM; m.S0 = x.S0; m.mu = x.mu; m.sigma = x.sigma;
        } else if constexpr (std::is_same_v<T, HestonParams>) {
            m.kind = MCQ_MODEL_HESTON; m.S0 = x.S0; m.mu = x.mu; m.kappa = x.kappa; m.theta = x.theta;
            m.xi = x.xi; m.rho = x.rho; m.v0 = x.v0; m.hes_L10 = x.L[1][0]; m.hes_L11 = x.L[1][1];
        } else if constexpr (std::is_same_v<T, DupireLocalParams>) {
            m.kind = MCQ_MODEL_DUPIRE; m.S0 = x.S0; m.mu = x.mu; m.sigma0 = x.sigma0; m.alpha = x.alpha;
            m.beta_d = x.beta_d; m.sigma = x.sigma0;
        } else {
            m.kind = MCQ_MODEL_MULTI_DUPIRE; m.n_assets = x.n; m.mu = x.mu; m.sigma0 = x.sigma0;
            m.alpha = x.alpha; m.beta_d = x.beta_d; m.uncorrelated = x.uncorrelated ? 1 : 0;
            m.S0_vec = x.S0.data(); m.S0 = x.S0.empty() ? 100.0 : x.S0[0];
            m.L = (x.uncorrelated || x.L.empty()) ? nullptr : x.L.data();
        }
    }, mv);
    return m;
}

inline mcq_payoff to_c(const PayoffVariant& pv) {
    mcq_payoff p{};
    std::visit([&](const auto& x) {
        using T = std::decay_t<decltype(x)>;
        if constexpr (std::is_same_v<T, European>) { p.kind = MCQ_PAYOFF_EUROPEAN; p.K = x.K; p.r = x.r; p.T = x.T; }
        else if constexpr (std::is_same_v<T, Asian>) { p.kind = MCQ_PAYOFF_ASIAN; p.K = x.K; }
        else if constexpr (std::is_same_v<T, GeomAsian>) { p.kind = MCQ_PAYOFF_GEOM_ASIAN; p.K = x.K; }
        else if constexpr (std::is_same_v<T, Lookback>) { p.kind = MCQ_PAYOFF_LOOKBACK; p.sigma = x.sigma; }
        else if constexpr (std::is_same_v<T, Barrier>) {
            p.kind = MCQ_PAYOFF_BARRIER_UP_OUT; p.K = x.K; p.B = x.B; p.sigma = x.sigma; p.r = x.r; p.T = x.T;
        } else { p.kind = MCQ_PAYOFF_BASKET; p.K = x.K; p.r = x.r; p.T = x.T; p.n_assets = x.n_assets; }
    }, pv);
    return p;
}

inline MCResult to_result(const mcq_result& r) { return {r.price, r.std_error, (long long)r.n_samples, r.time_s}; }
inline mcq_mc_cfg c_cfg(const MCConfig& c) {
    mcq_mc_cfg o; mcq_default_cfgs(&o, nullptr, nullptr);
    o.N_batch = c.N_batch; o.pilot_n = c.pilot_n; o.seed = c.seed;
    return o;
}
inline mcq_qmc_cfg c_cfg(const QMCConfig& c) {
    mcq_qmc_cfg o; mcq_default_cfgs(nullptr, &o, nullptr);
    o.R = c.R; o.max_doublings = c.max_doublings;
    return o;
}
inline mcq_mlmc_cfg c_cfg(const MLMCConfig& c) {
    mcq_mlmc_cfg o; mcq_default_cfgs(nullptr, nullptr, &o);
    o.M = c.M; o.max_L = c.max_L; o.pilot_n = c.pilot_n;
    return o;
}

}  // namespace mcq_detail

inline DeviceBBData* bb_upload(const BBData& bb) {
    auto* d = new DeviceBBData{nullptr, bb.N};
    const int rc = mcq_bb_create(bb.N, bb.T, &d->h);
    if (rc != MCQ_OK) { delete d; mcq_detail::check(rc); }
    return d;
}
inline void bb_free(DeviceBBData* d) {
    if (!d) return;
    mcq_handle_free(d->h);
    delete d;
}
inline DevicePCAData* pca_upload(const PCAData& pca) {
    auto* d = new DevicePCAData{nullptr, pca.m};
    const int rc = mcq_pca_create_from(pca.m, pca.T, pca.M_pca.data(), &d->h);
    if (rc != MCQ_OK) { delete d; mcq_detail::check(rc); }
    return d;
}
inline void pca_free(DevicePCAData* d) {
    if (!d) return;
    mcq_handle_free(d->h);
    delete d;
}

inline MCResult run_mc_cuda(const ModelVariant& model, const PayoffVariant& payoff, double eps, int n_steps,
                            const MCConfig& cfg = {}) {
    mcq_model m = mcq_detail::to_c(model);
    mcq_payoff p = mcq_detail::to_c(payoff);
    mcq_mc_cfg c = mcq_detail::c_cfg(cfg);
    mcq_result r{};
    mcq_detail::check(mcq_run_mc(&m, &p, eps, n_steps, &c, &r));
    return mcq_detail::to_result(r);
}

inline MCResult run_mlmc_cuda(const ModelVariant& model, const PayoffVariant& payoff, double eps,
                              const MLMCConfig& cfg = {}) {
    mcq_model m = mcq_detail::to_c(model);
    mcq_payoff p = mcq_detail::to_c(payoff);
    mcq_mlmc_cfg c = mcq_detail::c_cfg(cfg);
    mcq_result r{};
    mcq_detail::check(mcq_run_mlmc(&m, &p, eps, &c, &r));
    return mcq_detail::to_result(r);
}

inline MCResult run_qmc_cuda(const ModelVariant& model, const PayoffVariant& payoff, double eps, int n_steps,
                             const QMCConfig& cfg = {}, NoiseMode mode = NoiseMode::Raw,
                             DeviceBBData* dev_bb = nullptr, DevicePCAData* dev_pca = nullptr) {
    mcq_model m = mcq_detail::to_c(model);
    mcq_payoff p = mcq_detail::to_c(payoff);
    mcq_qmc_cfg c = mcq_detail::c_cfg(cfg);
    mcq_result r{};
    mcq_detail::check(mcq_run_qmc(&m, &p, eps, n_steps, &c, (int)mode, dev_bb ? dev_bb->h : nullptr,
                                  dev_pca ? dev_pca->h : nullptr, &r));
    return mcq_detail::to_result(r);
}

inline MCResult run_mlqmc_cuda(const ModelVariant& model, const PayoffVariant& payoff, double eps,
                               const MLMCConfig& ml_cfg = {}, const QMCConfig& qmc_cfg = {},
                               NoiseMode mode = NoiseMode::Raw, std::vector<DeviceBBData*> bb_list = {},
                               std::vector<DevicePCAData*> pca_list = {}) {
    mcq_model m = mcq_detail::to_c(model);
    mcq_payoff p = mcq_detail::to_c(payoff);
    mcq_mlmc_cfg ml = mcq_detail::c_cfg(ml_cfg);
    mcq_qmc_cfg qc = mcq_detail::c_cfg(qmc_cfg);
    std::vector<mcq_handle> bl, pl;
    for (auto* b : bb_list) bl.push_back(b ? b->h : nullptr);
    for (auto* q : pca_list) pl.push_back(q ? q->h : nullptr);
    mcq_result r{};
    mcq_detail::check(mcq_run_mlqmc(&m, &p, eps, &ml, &qc, (int)mode, bl.data(), (int)bl.size(), pl.data(),
                                    (int)pl.size(), &r));
    return mcq_detail::to_result(r);
}

inline CVPilot cv_pilot(const ModelVariant& main_model, const ModelVariant& ctrl_model,
                        const PayoffVariant& main_payoff, const PayoffVariant& ctrl_payoff, double E_ctrl,
                        int n_steps, int N_pilot, unsigned seed = 0) {
    mcq_model mm = mcq_detail::to_c(main_model), cm = mcq_detail::to_c(ctrl_model);
    mcq_payoff mp = mcq_detail::to_c(main_payoff), cp = mcq_detail::to_c(ctrl_payoff);
    mcq_cv_pilot_out o{};
    mcq_detail::check(mcq_cv_pilot(&mm, &cm, &mp, &cp, E_ctrl, n_steps, N_pilot, seed, &o));
    return {o.beta, o.var_plain, o.var_cv};
}

inline MCResult run_mc_cv_cuda(const ModelVariant& main_model, const ModelVariant& ctrl_model,
                               const PayoffVariant& main_payoff, const PayoffVariant& ctrl_payoff, double E_ctrl,
                               double beta, double eps, int n_steps, const MCConfig& cfg = {}) {
    mcq_model mm = mcq_detail::to_c(main_model), cm = mcq_detail::to_c(ctrl_model);
    mcq_payoff mp = mcq_detail::to_c(main_payoff), cp = mcq_detail::to_c(ctrl_payoff);
    mcq_mc_cfg c = mcq_detail::c_cfg(cfg);
    mcq_result r{};
    mcq_detail::check(mcq_run_mc_cv(&mm, &cm, &mp, &cp, E_ctrl, beta, eps, n_steps, &c, &r));
    return mcq_detail::to_result(r);
}

inline MCResult run_qmc_cv_cuda(const ModelVariant& main_model, const ModelVariant& ctrl_model,
                                const PayoffVariant& main_payoff, const PayoffVariant& ctrl_payoff, double E_ctrl,
                                double beta, double eps, int n_steps, const QMCConfig& cfg = {}) {
    mcq_model mm = mcq_detail::to_c(main_model), cm = mcq_detail::to_c(ctrl_model);
    mcq_payoff mp = mcq_detail::to_c(main_payoff), cp = mcq_detail::to_c(ctrl_payoff);
    mcq_qmc_cfg c = mcq_detail::c_cfg(cfg);
    mcq_result r{};
    mcq_detail::check(mcq_run_qmc_cv(&mm, &cm, &mp, &cp, E_ctrl, beta, eps, n_steps, &c, &r));
    return mcq_detail::to_result(r);
}

inline MCResult run_is_cuda(const GBMParams& model, const European& payoff, double z_star, double eps,
                            const MCConfig& cfg = {}) {
    mcq_model m = mcq_detail::to_c(ModelVariant(model));
    mcq_payoff p = mcq_detail::to_c(PayoffVariant(payoff));
    mcq_mc_cfg c = mcq_detail::c_cfg(cfg);
    mcq_result r{};
    mcq_detail::check(mcq_run_is(&m, &p, z_star, eps, &c, &r));
    return mcq_detail::to_result(r);
}

inline std::pair<double, double> run_mc_fixed(const ModelVariant& model, const PayoffVariant& payoff, int n_steps,
                                              long long n_paths, unsigned seed) {
    mcq_model m = mcq_detail::to_c(model);
    mcq_payoff p = mcq_detail::to_c(payoff);
    double mean = 0.0, var = 0.0;
    mcq_detail::check(mcq_run_mc_fixed(&m, &p, n_steps, n_paths, seed, &mean, &var));
    return {mean, var};
}
