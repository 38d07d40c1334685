/*
 * oracle.h — CPU oracle for the pricing hot path.  TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithm (QuantGuy3/financial-derivatives-
 * montecarlo), used only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference leg, and only as the checker or the timed CPU baseline.  The product library
 * (financial-derivatives-montecarlo_b200/) never links, loads or calls anything here.
 *
 * Each function cites the reference file:line it restates.  Pinning: the closed forms are
 * checked against the reference's published known answers (bs_call = 10.450584 and
 * 0.028643, informes_finales/informe_final.txt:7,158); the inverse normal against
 * scipy.special.ndtri; Philox against the Random123 known-answer vectors; the Sobol-HH
 * integer stream against the reference's own hh_scramble compiled from its source
 * (oracle/ref/, fixtures in tests/golden/).
 */
#ifndef MCQ_ORACLE_H
#define MCQ_ORACLE_H
#include <stdint.h>
#include "../include/mcq.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Sobol + Hong–Hickernell scrambling (methods_cuda.cu:753-825) ---- */
uint32_t orc_splitmix32(uint32_t x);
uint32_t orc_hh_scramble(uint32_t raw, uint32_t base);   /* row-by-row popcount form */
uint32_t orc_hh_linear(uint32_t v, uint32_t base);       /* same without the digital shift */
int      orc_dirvectors(const uint32_t** table);         /* JoeKuo6 via cuRAND; returns #dims */
uint32_t orc_sobol_raw(const uint32_t* v32, uint32_t n); /* curand Sobol32 after skipahead(n) */
/* literal restatement: raw via gray code, then hh_scramble per point */
void orc_sobol_hh_u32_literal(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n,
                              uint32_t* out);
/* fast form: pre-scrambled direction words + gray-code recurrence (bit-identical) */
void orc_sobol_hh_u32(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n,
                      uint32_t* out);
float  orc_u_of(uint32_t scrambled, int flags);          /* ((float)s + 1) * 2^-32 */
double orc_ppnd16(double p);                             /* Wichura AS241 inverse normal */
void   orc_sobol_hh_normal(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n,
                           int flags, double* out);

/* ---- Philox4x32-10 (Salmon et al. 2011) + Box–Muller ---- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_philox_normals(uint32_t seed, uint32_t stream, uint64_t path, int n, double* z);

/* ---- Brownian bridge (utils.cpp:54-124) ---- */
int  orc_bb_precompute(int N, double T, int* map_idx, int* left_idx, int* right_idx,
                       double* wl, double* wr, double* sd);
void orc_bb_apply(int N, const int* map_idx, const int* left_idx, const int* right_idx,
                  const double* wl, const double* wr, const double* sd,
                  const double* z, double* dW);

/* ---- PCA (utils.cpp:131-167) ---- */
int orc_pca_compute(int m, double T, double* M_colmajor);  /* closed-form eigenpairs */
int orc_pca_jacobi(int m, double T, double* M_colmajor);   /* numeric cross-check */

/* ---- closed forms (utils.cpp:22-47) ---- */
double orc_bs_call(double S0, double K, double T, double r, double sigma);
double orc_geom_asian(double S0, double K, double T, double mu, double sigma, int n);
double orc_down_out_call(double S0, double K, double B, double T, double r, double sigma);

/* ---- path arithmetic in FP64 (methods_cuda.cu:270-352, 388-551) ----
 * z: normals of one path in Sobol-dimension order (dim = step * d_noise + factor);
 * noise: MCQ_NOISE_*; bb/pca tables as produced above (may be NULL for RAW);
 * pca_fp16: round z and M to binary16 before the product (methods_cuda.cu:1228). */
typedef struct orc_noise {
    int mode;
    int N;
    const int *map_idx, *left_idx, *right_idx;
    const double *wl, *wr, *sd;
    const double* M_pca;   /* column-major N x N */
    int pca_fp16;
} orc_noise;

int    orc_noise_dim(const mcq_model* m);
double orc_path_payoff(const mcq_model* m, const mcq_payoff* p, int n_steps,
                       const orc_noise* nz, const double* z);
double orc_path_payoff_f(const mcq_model* m, const mcq_payoff* p, int n_steps,
                         const orc_noise* nz, const double* z, int flags);
/* coupled fine/coarse pair (kernel_mlmc, methods_cuda.cu:445-518): returns Yf, *yc = Yc */
double orc_level_payoff(const mcq_model* m, const mcq_payoff* p, int n_fine, int M,
                        const orc_noise* nz, const double* z, int flags, double* yc);

/* coupled correlated GBM basket call with pathwise d(dY)/dS0_a in dd[n_assets]; M <= 0: level 0 */
double orc_basket_level(const mcq_model* m, const mcq_payoff* p, int n_fine, int M, const double* z,
                        double* yc, double* dd);
double orc_basket_level_f(const mcq_model* m, const mcq_payoff* p, int n_fine, int M, const double* z,
                          double* yc, double* dd, int flags);

/* ---- drivers (sums over replicas/points; OpenMP) ---- */
/* sums[R][2]: {sum Y, sum Y^2} over points offset..offset+N-1 of salts salt_base + r */
int orc_qmc_sums(const mcq_model* m, const mcq_payoff* p, int n_steps, const orc_noise* nz,
                 uint32_t salt_base, int R, uint32_t offset, int64_t N, int flags,
                 int n_threads, double* sums);
/* sums[R][4]: {sum dY, sum dY^2, sum Yf, sum Yf^2}; use_sobol=0 -> Philox(seed, stream) */
int orc_level_sums(const mcq_model* m, const mcq_payoff* p, int n_fine, int M,
                   const orc_noise* nz, int use_sobol, uint32_t seed, uint32_t salt_base,
                   int R, uint32_t offset, int64_t N, int flags, int n_threads, double* sums);
/* sums[R][4 + n]: {sum dY, sum dY^2, sum Yf, sum Yf^2, sum d(dY)/dS0_a ...} over scrambled
   Sobol points offset..offset+N-1 of salts salt_base + r (basket model, raw ordering) */
int orc_basket_level_sums(const mcq_model* m, const mcq_payoff* p, int n_fine, int M, uint32_t salt_base,
                          int R, uint32_t offset, int64_t N, int flags, int n_threads, double* sums);
/* sums[2] over Philox paths first_path .. first_path + n_paths - 1 of (seed, stream) */
/* kernel_is_gbm (methods_cuda.cu:685-707) in FP64: per-replica IS sums over scrambled Sobol or
   Philox normals; z_star is the per-step drift shift. */
double orc_is_payoff(const mcq_model* m, const mcq_payoff* p, int n_steps, double z_star, const double* z);
int orc_is_sums(const mcq_model* m, const mcq_payoff* p, int n_steps, double z_star, int use_sobol,
                uint32_t seed, uint32_t salt_base, int R, uint32_t offset, int64_t N, int flags,
                int n_threads, double* sums);
int orc_mc_sums(const mcq_model* m, const mcq_payoff* p, int n_steps, uint32_t seed,
                uint32_t stream, int64_t first_path, int64_t n_paths, int n_threads,
                double* sums);

/* adaptive RQMC driver restated from run_qmc_cuda (methods_cuda.cu:1624-1668) */
int orc_run_qmc(const mcq_model* m, const mcq_payoff* p, double eps, int n_steps,
                const orc_noise* nz, int R, int max_doublings, int64_t N0,
                uint32_t salt_base, int flags, int n_threads, mcq_result* out);

int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
