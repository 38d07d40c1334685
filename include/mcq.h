/*
 * mcq.h — C ABI of the B200-native MC / RQMC / MLMC / MLQMC pricing engine.
 *
 * Every entry point is `extern "C"`, takes plain structs, pointers and sizes, returns an
 * int status (MCQ_OK == 0) and never lets a C++ exception escape.  On failure the status
 * is non-zero and mcq_last_error() returns a thread-local message.
 *
 * The entry points replace the reference's C++ driver API (methods_cuda.cuh:58-134 of
 * QuantGuy3/financial-derivatives-montecarlo); each declaration below names the
 * reference function it stands in for.  include/mcq.hpp layers the reference's own C++
 * types (ModelVariant, PayoffVariant, MCConfig, ...) over this ABI so that callers of the
 * reference compile unchanged.
 *
 * Conventions
 *   - Output buffers are caller-owned.  Host pointers unless the name says "device".
 *   - `stream` arguments are cudaStream_t passed as void*; NULL means the engine's own
 *     internal stream.
 *   - The engine uses the CUDA device selected by mcq_init() (default: current device).
 *   - Not re-entrant per handle: two threads must not share one BB/PCA handle at the same
 *     time.  Distinct handles may be used concurrently.
 */
#ifndef MCQ_H
#define MCQ_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
#define MCQ_OK               0
#define MCQ_ERR_INVALID      1   /* bad argument (size, kind, null pointer)          */
#define MCQ_ERR_CUDA         2   /* a CUDA runtime call failed                       */
#define MCQ_ERR_UNSUPPORTED  3   /* combination the engine does not implement        */
#define MCQ_ERR_RANGE        4   /* Sobol offset beyond 2^32, dimension beyond table */
#define MCQ_ERR_NOMEM        5   /* device or host allocation failed                 */
#define MCQ_ERR_INTERNAL     6
#define MCQ_ERR_TIMEOUT      7   /* a bounded device-side wait gave up               */

/* ---------------------------------------------------------------- enumerations */
/* Model kinds.  0..3 follow ModelKind (methods_cuda.cu:205); 4, 5 are engine additions. */
#define MCQ_MODEL_GBM            0  /* GBMParams          models.hpp:15-21 */
#define MCQ_MODEL_HESTON         1  /* HestonParams       models.hpp:23-43 */
#define MCQ_MODEL_DUPIRE         2  /* DupireLocalParams  models.hpp:45-54 */
#define MCQ_MODEL_MULTI_DUPIRE   3  /* MultiDupireParams  models.hpp:56-68 */
#define MCQ_MODEL_LOCALVOL_GRID  4  /* grid local-vol surface, bilinear (new)            */
#define MCQ_MODEL_BASKET_GBM     5  /* correlated GBM basket, per-asset sigma (new)      */

/* Payoff kinds.  0..5 follow PayoffKind (methods_cuda.cu:202); 6 is an engine addition. */
#define MCQ_PAYOFF_EUROPEAN          0  /* payoffs.hpp:14 */
#define MCQ_PAYOFF_ASIAN             1  /* payoffs.hpp:15 (undiscounted, as the reference) */
#define MCQ_PAYOFF_GEOM_ASIAN        2  /* payoffs.hpp:16 (undiscounted) */
#define MCQ_PAYOFF_LOOKBACK          3  /* payoffs.hpp:17 floating strike, undiscounted */
#define MCQ_PAYOFF_BARRIER_UP_OUT    4  /* payoffs.hpp:18 */
#define MCQ_PAYOFF_BASKET            5  /* payoffs.hpp:19 */
#define MCQ_PAYOFF_BARRIER_DOWN_OUT  6  /* down-and-out call (new) */

/* Noise transforms (NoiseMode, methods_cuda.cuh:35). */
#define MCQ_NOISE_RAW  0
#define MCQ_NOISE_BB   1
#define MCQ_NOISE_PCA  2

/* Behaviour flags (mcq_qmc_cfg.flags / mcq_mlmc_cfg.flags). */
#define MCQ_FLAG_COMPAT_U_INF        1  /* keep u = 1.0f -> +inf normal (methods_cuda.cu:823);
                                           default maps that single float to 1 - 2^-24 */
#define MCQ_FLAG_COMPAT_HESTON_MLMC  2  /* skip the running (path-dependent) update on the
                                           Heston coupled path, as methods_cuda.cu:464-490 */
#define MCQ_FLAG_HESTON_MILSTEIN     8  /* Heston variance step with the Milstein term
                                           xi^2/4 (dW2^2 - h) (Euler-Milstein, full truncation);
                                           default: the reference's Euler step (:276-284) */
#define MCQ_FLAG_BASKET_OWN_S0      16  /* Dupire basket: scale each asset's local volatility
                                           by its own S0, sigma0 e^{-alpha t} (S_a / S0_a)^(beta-1);
                                           default: asset 0's S0 for every asset, as the
                                           reference (c_p.S0 = S0[0], methods_cuda.cu:1046, :538-542) */

/* ---------------------------------------------------------------- parameter structs */
typedef struct mcq_model {
    int32_t kind;                 /* MCQ_MODEL_* */
    int32_t n_assets;             /* MULTI_DUPIRE / BASKET_GBM */
    /* common */
    double S0, mu, T;
    /* GBM */
    double sigma;
    /* Heston: dS = mu S dt + sqrt(v) S dW1, dv = kappa(theta - v) dt + xi sqrt(v) dW2.
       hes_L10/hes_L11 are the second row of the 2x2 Cholesky factor exactly as
       HestonParams::L (models.hpp:36-42); mcq_model_heston() fills them from rho. */
    double kappa, theta, xi, rho, v0, hes_L10, hes_L11;
    /* parametric Dupire: sigma_loc = sigma0 exp(-alpha t) (S/S0)^(beta_d - 1) */
    double sigma0, alpha, beta_d;
    /* multi-asset */
    int32_t uncorrelated;         /* 1: rho = I, L ignored */
    int32_t _pad0;
    const double* S0_vec;         /* [n_assets] */
    const double* L;              /* [n_assets * n_assets] row-major lower Cholesky */
    const double* sigma_vec;      /* [n_assets] BASKET_GBM */
    const double* weights;        /* [n_assets] BASKET_GBM (NULL: equal weights) */
    /* local-vol grid: sigma(K_i, t_j) at lv_sigma[j * lv_nK + i] */
    int32_t lv_nK, lv_nt;
    const double* lv_K;           /* [lv_nK] increasing */
    const double* lv_t;           /* [lv_nt] increasing */
    const double* lv_sigma;       /* [lv_nt * lv_nK] */
} mcq_model;

typedef struct mcq_payoff {
    int32_t kind;                 /* MCQ_PAYOFF_* */
    int32_t n_assets;             /* Basket{... n_assets} */
    double K, B, r, T, sigma;     /* sigma: BGK continuity-correction volatility (Lookback, Barrier) */
} mcq_payoff;

/* MCConfig (methods_cuda.cuh:10-14). */
typedef struct mcq_mc_cfg {
    int64_t  N_batch;             /* default 1<<16; only bounds host bookkeeping here */
    int32_t  pilot_n;             /* default 10000 */
    uint32_t seed;                /* default 123 */
} mcq_mc_cfg;

/* QMCConfig (methods_cuda.cuh:16-26) plus the values the reference hard-codes. */
typedef struct mcq_qmc_cfg {
    int32_t  R;                   /* default 32 replicas */
    int32_t  max_doublings;       /* default 20 */
    int64_t  N0_per_replica;      /* 0: the reference's memory-derived start (methods_cuda.cu:1523-1533) */
    uint32_t salt_base;           /* default 42 (methods_cuda.cu:1564) */
    int32_t  flags;               /* MCQ_FLAG_* */
} mcq_qmc_cfg;

/* MLMCConfig (methods_cuda.cuh:28-32) plus the level-0 step count. */
typedef struct mcq_mlmc_cfg {
    int32_t M;                    /* default 2 */
    int32_t max_L;                /* default 10 */
    int32_t pilot_n;              /* default 400 */
    int32_t n0_steps;             /* steps on level 0; the reference uses 1 (methods_cuda.cu:1349) */
    int32_t flags;                /* MCQ_FLAG_* */
    uint32_t seed;                /* MLMC pseudo-random stream base; default 42 (methods_cuda.cu:1412) */
} mcq_mlmc_cfg;

/* MCResult (methods_cuda.cuh:42-47) plus work accounting. */
typedef struct mcq_result {
    double  price;
    double  std_error;
    int64_t n_samples;
    double  time_s;
    double  path_steps;           /* total simulated path-steps (fine + coarse for MLMC) */
    int32_t levels;               /* MLMC/MLQMC: L + 1 */
    int32_t launches;             /* engine kernel launches issued */
    int32_t converged;            /* 1: the driver's stopping test passed (MLMC/MLQMC: the bias
                                     test before the iteration cap, :1473 / :1999; QMC: var of
                                     the replica means < eps^2/2 before the doubling cap); MC, CV
                                     and IS size N from the pilot and always report 1 */
    int32_t reserved;
} mcq_result;

/* CVPilot (methods_cuda.cuh:94). */
typedef struct mcq_cv_pilot_out { double beta, var_plain, var_cv; } mcq_cv_pilot_out;

/* Pathwise adjoint Greeks (mcq_adjoint). */
typedef struct mcq_greeks {
    double price, delta, rho, vega;               /* means over all R x n_points paths */
    double price_se, delta_se, rho_se, vega_se;   /* standard errors from the R replica means */
    int64_t n_paths;
    int32_t n_nodes;                              /* grid nodes written to node_vega (0 otherwise) */
    int32_t launches;
    double  time_s;
    double  path_steps;                           /* forward + recompute + reverse path-steps */
} mcq_greeks;

/* One option of a batched book (mcq_book_price), priced by MLQMC to its own eps.  Either
   (model == NULL) a call on a weighted basket of correlated GBM assets,
   max(sum_a w_a S_a(T) - K, 0) e^{-rT}, drift r, with the pathwise delta per asset; or
   (model != NULL) a single-asset option: `model` (GBM, Heston or parametric Dupire; its T is the
   maturity) with `payoff` (European, Asian, geometric Asian, lookback, up- or down-and-out
   barrier), the coupled level pair of mcq_run_mlqmc; then n_assets, K, r, T, S0, sigma, weights
   and L are not read and no deltas are returned.  No counterpart in the reference. */
#define MCQ_BOOK_MAX_ASSETS 16
typedef struct mcq_book_option {
    int32_t n_assets;             /* 1..16 */
    int32_t max_L;                /* finest level, 2..11; level l has n0_steps * M^l steps */
    double K, r, T, eps;
    const double* S0;             /* [n_assets] */
    const double* sigma;          /* [n_assets] */
    const double* weights;        /* [n_assets]; NULL: equal weights */
    const double* L;              /* [n_assets^2] row-major lower Cholesky; NULL: uncorrelated */
    const mcq_model* model;       /* NULL: the basket above; else a single-asset model */
    const mcq_payoff* payoff;     /* the single-asset option's payoff (with model) */
} mcq_book_option;

typedef struct mcq_book_result {
    double  price, std_error;     /* sum over levels of the level means; SE as run_mlqmc */
    double  delta[MCQ_BOOK_MAX_ASSETS];   /* pathwise d price / d S0_a, first n_assets used */
    int64_t n_samples;            /* sum over levels of N_l x R */
    int32_t levels;               /* L + 1 */
    int32_t converged;            /* 1: the bias test passed before the iteration cap */
} mcq_book_result;

typedef struct mcq_book_stats {
    double  time_s;               /* pricing time, after the per-book set-up */
    double  setup_s;              /* parameter upload and scrambled tables */
    double  path_steps;           /* sum over slices of R x points x (fine + coarse steps) */
    double  normals;              /* sum over slices of R x points x fine steps x assets */
    int32_t rounds;               /* adaptive rounds (batched) / per-option steps (plain) */
    int32_t launches;             /* kernel launches issued */
} mcq_book_stats;

#define MCQ_BOOK_BATCHED  0       /* every option and level in one graph replay per round */
#define MCQ_BOOK_PLAIN    1       /* one option at a time, one launch per level on its stream */

typedef struct mcq_handle_s* mcq_handle;   /* opaque BB / PCA handle */

/* ---------------------------------------------------------------- lifecycle */
int         mcq_init(int device);          /* -1: current device */
int         mcq_shutdown(void);
const char* mcq_last_error(void);
int         mcq_version(void);             /* major*10000 + minor*100 + patch */
int         mcq_default_cfgs(mcq_mc_cfg* mc, mcq_qmc_cfg* qmc, mcq_mlmc_cfg* ml);
int         mcq_model_heston(double S0, double mu, double kappa, double theta, double xi,
                             double rho, double v0, double T, mcq_model* out);

/* ---------------------------------------------------------------- BB / PCA handles
 * mcq_bb_create   replaces bb_precompute + bb_upload   (utils.cpp:54-101, methods_cuda.cu:928-953)
 * mcq_pca_create  replaces pca_compute  + pca_upload   (utils.cpp:131-167, methods_cuda.cu:962-971)
 * mcq_pca_create_from uploads a caller-supplied m x m column-major M_pca.
 * mcq_handle_free replaces bb_free / pca_free          (methods_cuda.cu:955-977) */
int mcq_bb_create(int N, double T, mcq_handle* out);
int mcq_pca_create(int m, double T, mcq_handle* out);
int mcq_pca_create_from(int m, double T, const double* M_pca_colmajor, mcq_handle* out);
int mcq_handle_free(mcq_handle h);
int mcq_handle_info(mcq_handle h, int* kind, int* n);

/* ---------------------------------------------------------------- estimator drivers */
/* run_mc_cuda (methods_cuda.cu:1272-1298): pilot, N = 2 Var / eps^2, main run. */
int mcq_run_mc(const mcq_model* m, const mcq_payoff* p, double eps, int n_steps,
               const mcq_mc_cfg* cfg, mcq_result* out);
/* run_mc_fixed (methods_cuda.cu:2368-2374): mean and variance of the mean of n_paths. */
int mcq_run_mc_fixed(const mcq_model* m, const mcq_payoff* p, int n_steps, int64_t n_paths,
                     uint32_t seed, double* mean, double* var_of_mean);
/* run_qmc_cuda (methods_cuda.cu:1494-1673): R scrambled replicas, doubling. */
int mcq_run_qmc(const mcq_model* m, const mcq_payoff* p, double eps, int n_steps,
                const mcq_qmc_cfg* cfg, int noise_mode, mcq_handle bb, mcq_handle pca,
                mcq_result* out);
/* run_mlmc_cuda (methods_cuda.cu:1305-1487). */
int mcq_run_mlmc(const mcq_model* m, const mcq_payoff* p, double eps,
                 const mcq_mlmc_cfg* cfg, mcq_result* out);
/* run_mlqmc_cuda (methods_cuda.cu:1680-2019); bb_list/pca_list: one handle per level. */
int mcq_run_mlqmc(const mcq_model* m, const mcq_payoff* p, double eps,
                  const mcq_mlmc_cfg* ml, const mcq_qmc_cfg* qmc, int noise_mode,
                  const mcq_handle* bb_list, int n_bb, const mcq_handle* pca_list, int n_pca,
                  mcq_result* out);
/* cv_pilot (methods_cuda.cu:2026-2076). */
int mcq_cv_pilot(const mcq_model* main_m, const mcq_model* ctrl_m, const mcq_payoff* main_p,
                 const mcq_payoff* ctrl_p, double E_ctrl, int n_steps, int N_pilot,
                 uint32_t seed, mcq_cv_pilot_out* out);
/* run_mc_cv_cuda (methods_cuda.cu:2078-2163). */
int mcq_run_mc_cv(const mcq_model* main_m, const mcq_model* ctrl_m, const mcq_payoff* main_p,
                  const mcq_payoff* ctrl_p, double E_ctrl, double beta, double eps, int n_steps,
                  const mcq_mc_cfg* cfg, mcq_result* out);
/* run_qmc_cv_cuda (methods_cuda.cu:2165-2278). */
int mcq_run_qmc_cv(const mcq_model* main_m, const mcq_model* ctrl_m, const mcq_payoff* main_p,
                   const mcq_payoff* ctrl_p, double E_ctrl, double beta, double eps, int n_steps,
                   const mcq_qmc_cfg* cfg, mcq_result* out);
/* run_is_cuda (methods_cuda.cu:2285-2365): GBM European with drift shift z_star. */
int mcq_run_is(const mcq_model* gbm, const mcq_payoff* european, double z_star, double eps,
               const mcq_mc_cfg* cfg, mcq_result* out);

/* ---------------------------------------------------------------- sensitivities
 * Pathwise adjoint Greeks over R scrambled-Sobol replicas (salts salt_base + r, points offset ..
 * offset + n_points - 1); no counterpart in the reference, which computes no Greeks.
 * delta = dV/dS0, rho = dV/d(rate) with the drift mu and the payoff's discount rate moving
 * together, vega = dV/dsigma (GBM), dV/dsigma0 (parametric Dupire), the parallel shift of the
 * local-vol grid, or dV/dv0 (Heston; full-truncation subgradient where V <= 0, and the Milstein
 * step with MCQ_FLAG_HESTON_MILSTEIN); node_vega (optional, lv_nt * lv_nK doubles, same layout
 * as lv_sigma) receives dV/dsigma(K_i, t_j).  Lipschitz payoffs only: European, arithmetic Asian,
 * lookback.  n_steps: multiple of 32 in [32, 1024] (Heston: of 16 in [16, 1024]); path states
 * are checkpointed every 16 steps and recomputed in the reverse sweep. */
int mcq_adjoint(const mcq_model* m, const mcq_payoff* p, int n_steps, uint32_t salt_base, int R,
                uint32_t offset, int64_t n_points, int flags, mcq_greeks* out, double* node_vega);

/* Batched book: prices n options by MLQMC (the adaptive level / sample logic of
 * run_mlqmc_cuda, methods_cuda.cu:1950-2000, per option; R = qc->R replicas with salts
 * qc->salt_base + l R + r; M, pilot_n, n0_steps from ml; ml->max_L is ignored in favour of
 * each option's own).  MCQ_BOOK_BATCHED runs every option's pending slices of a round in one
 * persistent work-queue kernel replayed from a CUDA graph; MCQ_BOOK_PLAIN is the per-option,
 * stream-per-level form (methods_cuda.cu:1745-1755) with the same kernels.  Both give
 * bit-identical results.  No counterpart in the reference (which rejects basket MLQMC,
 * methods_cuda.cu:1695-1697).  stats may be NULL. */
int mcq_book_price(const mcq_book_option* opts, int n, const mcq_mlmc_cfg* ml, const mcq_qmc_cfg* qc,
                   int mode, mcq_book_result* out, mcq_book_stats* stats);

/* The same book built up incrementally (the submit / run form of the batched path).  A book
 * object copies every option it is given (arrays included), so the caller's arrays may be freed
 * after mcq_book_submit returns.  mcq_book_run prices everything submitted so far, in
 * submission order, exactly as mcq_book_price; mcq_book_clear empties the book.  Not
 * re-entrant per book object. */
typedef struct mcq_book_s* mcq_book;
int mcq_book_create(mcq_book* out);
int mcq_book_submit(mcq_book b, const mcq_book_option* opts, int n);   /* appends n options */
int mcq_book_size(mcq_book b, int* n);
int mcq_book_run(mcq_book b, const mcq_mlmc_cfg* ml, const mcq_qmc_cfg* qc, int mode,
                 mcq_book_result* out, mcq_book_stats* stats);         /* out: one per option */
int mcq_book_clear(mcq_book b);
int mcq_book_free(mcq_book b);

/* ---------------------------------------------------------------- hot-path passes
 * One fused kernel pass over R replicas x n_points scrambled-Sobol points (salts
 * salt_base + r, point indices offset .. offset + n_points - 1).  sums_host receives
 * [R][2] doubles {sum Y, sum Y^2}.  This is the unit the QMC driver repeats per doubling
 * (accumulate_range, methods_cuda.cu:1549-1622, with no D x N array). */
int mcq_qmc_pass(const mcq_model* m, const mcq_payoff* p, int n_steps, int noise_mode,
                 mcq_handle bb, mcq_handle pca, uint32_t salt_base, int R, uint32_t offset,
                 int64_t n_points, int flags, double* sums_host);
/* Same pass with device-resident output (sums_device: R*2 doubles) on `stream`;
   asynchronous.  Used to time the kernel with inputs and outputs resident in HBM.  A bounded
   device-side wait that gives up in such a pass (MCQ_ERR_TIMEOUT) is reported by the next
   synchronous call on the engine's default workspace (mcq_qmc_pass, mcq_level_pass, mcq_run_qmc,
   mcq_run_mc). */
int mcq_qmc_pass_device(const mcq_model* m, const mcq_payoff* p, int n_steps, int noise_mode,
                        mcq_handle bb, mcq_handle pca, uint32_t salt_base, int R,
                        uint32_t offset, int64_t n_points, int flags, double* sums_device,
                        void* stream);
/* Pseudo-random (Philox4x32-10) pass over n_paths paths of stream `stream_id`, starting
   at path index first_path: sums_host[2] = {sum Y, sum Y^2}.  The unit behind run_mc. */
int mcq_mc_pass(const mcq_model* m, const mcq_payoff* p, int n_steps, uint32_t seed,
                uint32_t stream_id, int64_t first_path, int64_t n_paths, double* sums_host);
/* Coupled fine/coarse level pass (kernel_mlmc, methods_cuda.cu:445-518): sums_host receives
   [R][4] = {sum dY, sum dY^2, sum Yf, sum Yf^2}.  use_sobol=1: salts salt_base + r and
   offset; use_sobol=0: Philox with key `seed`, stream salt_base + r, paths from offset. */
int mcq_level_pass(const mcq_model* m, const mcq_payoff* p, int n_fine, int M, int noise_mode,
                   mcq_handle bb, mcq_handle pca, int use_sobol, uint32_t seed,
                   uint32_t salt_base, int R, uint32_t offset, int64_t n_points, int flags,
                   double* sums_host);

/* Importance-sampling pass (kernel_is_gbm, methods_cuda.cu:685-707): GBM European paths under
   the drift shift z_star_step per step (run_is_cuda passes z_star / sqrt(n_steps), :2297),
   payoff times the likelihood ratio; sums_host[R][2] = {sum Y, sum Y^2}.  use_sobol=1:
   scrambled Sobol with salts salt_base + r from point `offset`; 0: Philox key `seed`, stream
   salt_base + r.  The unit behind mcq_run_is (which uses Philox). */
int mcq_is_pass(const mcq_model* m, const mcq_payoff* p, int n_steps, double z_star_step, int use_sobol,
                uint32_t seed, uint32_t salt_base, int R, uint32_t offset, int64_t n_points, int flags,
                double* sums_host);

/* One RQMC pass (as mcq_qmc_pass_device) that allocates no device memory.  No counterpart in
 * the reference.  For callers that may not call cudaMalloc: code living in a process whose GPU
 * memory belongs to another allocator (a framework's caching allocator, a plugin host with a
 * fixed budget) and latency-critical paths where cudaMalloc / cudaFree would synchronise the
 * device.  Its scratch is one fixed __device__ array inside the library (about 2.7 MiB, held on
 * every GPU that loads the library until exit); sums_device ([R][2] doubles) is the caller's.
 * Limits: GBM, Heston or parametric Dupire, raw ordering, n_steps x factors <= 512, R <= 32;
 * larger requests fail with MCQ_ERR_RANGE.  Same kernel family, work split and carried Sobol
 * start words as mcq_qmc_pass_device (in one of the family's launch variants, which all give
 * the same bits), hence the same sums bit for bit.  The first call on a device (and the first in a new context of
 * it, e.g. after cudaDeviceReset) loads the direction table into the array with a synchronous
 * copy and should come before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race, so keep them on one stream.  Asynchronous on `stream` (NULL: the
 * legacy default stream). */
int mcq_qmc_pass_noalloc(const mcq_model* m, const mcq_payoff* p, int n_steps, uint32_t salt_base,
                         int R, uint32_t offset, int64_t n_points, int flags, double* sums_device,
                         void* stream);

/* ---------------------------------------------------------------- parity / debug exports
 * Hong–Hickernell scrambled Sobol stream (methods_cuda.cu:753-825): out[d * n + i] for
 * dimension dim0 + d and point index offset + i.  _u32 returns the scrambled integers,
 * _normal the N(0,1) values the path kernels consume. */
int mcq_sobol_hh_u32(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n,
                     uint32_t* out_host);
int mcq_sobol_hh_normal(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n,
                        int flags, float* out_host);
/* Failure-path probe: one warp waits `polls` (1 .. 2^20) times on a device barrier that nothing
   completes, as the bounded waits of the assisted and tensor-core passes do, and returns
   MCQ_ERR_TIMEOUT through the same status word; the context stays usable. */
int mcq_debug_wait_timeout(uint32_t polls);
/* Philox4x32-10 block (counter, key) -> 4 words; host-side, for known-answer checks. */
int mcq_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* BB / PCA tables as the device sees them (for parity tests). */
int mcq_bb_tables(mcq_handle bb, int* map_idx, float* wl, float* wr, float* sd);  /* per dimension */
int mcq_pca_matrix(mcq_handle pca, float* M_colmajor_f32);
/* The normals (raw) or time-ordered increments (bridge, PCA) that one fused pass consumed,
   for bit-level parity tests: out_host[R][n_points][n_steps * d_noise].  n_points <= 2^20.
   `bb` is the BB handle for MCQ_NOISE_BB and the PCA handle for MCQ_NOISE_PCA. */
int mcq_debug_pass_dump(const mcq_model* m, int n_steps, int noise_mode, mcq_handle bb,
                        int use_sobol, uint32_t seed, uint32_t salt_base, int R, uint32_t offset,
                        int64_t n_points, int flags, float* out_host);
/* Work layout of the last fused path-kernel launch of the allocating passes and drivers (not the
   tensor-core PCA pass, the book or mcq_qmc_pass_noalloc): the 32-point groups per work item and
   the Sobol start words each warp carries from group to group in shared memory (0: every tile
   walks its start word from the digital shift). */
int mcq_debug_last_pass_layout(int* groups_per_item, int* carry_words);
/* The book kernel's per-replica sums over one slice of one option (level `level`, points
   offset .. offset + n_points - 1, R = qc->R replicas with salts qc->salt_base + level R + r):
   sums_host[R][20] = {sum dY, sum dY^2, sum Yf, sum Yf^2, sum d(dY)/dS0_a for a < 16 (0 beyond
   n_assets)}.  For parity tests of the book against the oracle. */
int mcq_book_level_sums(const mcq_book_option* opt, const mcq_mlmc_cfg* ml, const mcq_qmc_cfg* qc, int level,
                        uint32_t offset, int64_t n_points, double* sums_host);

#ifdef __cplusplus
}
#endif
#endif /* MCQ_H */
