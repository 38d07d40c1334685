// kparams.h — parameter block shared by the host launch code and the device kernels.
//
// One KParams value describes one fused kernel pass: which generator, noise transform, model
// and payoff, the path geometry, the work split into warp items, and where the per-item
// partial sums go.  It replaces the reference's `__constant__ KernelParams c_p`
// (methods_cuda.cu:211-246): it travels by value as a __grid_constant__ kernel argument, so
// passes with different parameters can be in flight on different streams at the same time
// (the reference has to keep c_p level-independent for exactly that reason, :1322-1324).
#pragma once
#include <cstdint>
#include <vector_types.h>

namespace mcq {

enum Gen : int { GEN_SOBOL = 0, GEN_PHILOX = 1 };
// NOISE_PACKED: raw ordering for paths of at most 16 normals, 32 / D path groups per Sobol tile
// (an engine-internal choice, never requested through the API)
// NOISE_ASSIST: raw ordering for passes with few, long paths: each path-owning warp is fed its
// normal tiles by three helper warps (engine-internal as well)
// NOISE_BB_UNI: the Brownian bridge whose window weights are the same for every point of a level
// (read from KParams::bbw instead of the per-dimension table; engine-internal)
// NOISE_DW: time-ordered increments computed outside the pass (the PCA orderings whose factor does
// not fit the tensor-core kernel's shared memory), read from KParams::dw_in (engine-internal)
enum Noise : int { NOISE_RAW = 0, NOISE_BB = 1, NOISE_PCA = 2, NOISE_PACKED = 3, NOISE_ASSIST = 4, NOISE_BB_UNI = 5,
                   NOISE_DW = 6 };

// Status written to KParams::err when a bounded device wait gives up (MCQ_ERR_TIMEOUT).
constexpr int MCQ_ERR_TIMEOUT_CODE = 7;
// MCQ_FLAG_BASKET_OWN_S0 and MCQ_FLAG_COMPAT_U_INF as the kernels test them in KParams::flags.
constexpr int MCQ_FLAG_OWN_S0_CODE = 16;
constexpr int MCQ_FLAG_COMPAT_U_INF_CODE = 1;
enum ModelK : int { MOD_GBM = 0, MOD_HESTON = 1, MOD_DUPIRE = 2, MOD_MULTI = 3, MOD_LVGRID = 4, MOD_BASKET = 5 };
enum PayK : int { PAY_EUR = 0, PAY_ASIAN = 1, PAY_GEOM = 2, PAY_LOOKBACK = 3, PAY_UPOUT = 4, PAY_BASKET = 5, PAY_DOWNOUT = 6 };
enum Est : int { EST_PLAIN = 0, EST_COUPLED = 1, EST_CV_ASIAN = 2, EST_CV_DUPIRE = 3, EST_IS = 4 };

constexpr int kWarpsPerBlock = 8;
constexpr int kThreads = kWarpsPerBlock * 32;
constexpr int kMaxBasket = 16;          // register-resident basket width
constexpr int kMaxWideBasket = 128;     // wide baskets: per-asset state in local memory
constexpr int kMaxHugeBasket = 1024;    // widest (the reference's 1000-asset example)
constexpr int kMinBlocks = 3;           // resident CTAs per SM the register budget is set for
constexpr int kMaxStats = 8;
// Assisted passes (NOISE_ASSIST): per owner warp, three helper warps and a ring of four 32 x 32
// normal tiles with a `full` and an `empty` mbarrier per slot.
constexpr int kAssistSlots = 4;
constexpr int kAssistHelpers = 3;
constexpr int kAssistTeam = 1 + kAssistHelpers;              // warps per owner
constexpr int kAssistTeams = kWarpsPerBlock / kAssistTeam;   // owners per block
constexpr int kAssistTeamBytes = kAssistSlots * 1024 * 4 + 2 * kAssistSlots * 8;

struct KParams {
    // ---- geometry
    int gen, noise, model, payoff, est;
    int n_steps;        // fine steps
    int d_noise;        // normals per step
    int D;              // n_steps * d_noise (Sobol dimensions / normals per path)
    int M;              // coupling factor (EST_COUPLED); coarse step every M fine steps
    int n_coarse;       // 0 on level 0 (no coarse path)
    int flags;
    int nstat;
    // ---- work split: R replicas x [offset, offset + n_points) points in 32-point groups
    int R;
    int gpi;            // groups per item
    int carry;          // Sobol start-state words per warp in shared memory (0: walk every tile)
    int items_per_rep;
    int n_items;
    uint64_t offset;    // first point (Sobol index / Philox path id)
    uint64_t n_points;  // points per replica
    uint64_t g0;        // first group = offset >> 5
    uint64_t G;         // groups per replica
    // ---- model (single precision, as the reference's c_p)
    float S0, inv_S0, mu, T, h, sqrt_h, sigma;
    float kappa, theta, xi, L10, L11, v0, om_f;    // om_f = 1 - exp(-kappa h), from expm1
    float sigma0, alpha, bm1;                      // Dupire: bm1 = beta_d - 1
    float hc, om_c;                                // coarse step, 1 - exp(-kappa hc)
    float mil;                                     // Heston Milstein: xi^2/4 (0: Euler)
    // ---- payoff
    float K, B, disc, corr_f, corr_c, u_cap;
    float pay_T;                                   // payoff maturity (discount sensitivity)
    // ---- control variate / importance sampling
    float beta_cv, E_ctrl, z_star;
    float ctrl_sigma;                              // GBM control volatility (EST_CV_DUPIRE)
    // ---- basket: packed [S0 | sigma | weight | L(n x n row-major)], float
    int n_assets;
    int uncorrelated;
    const float* bsk;
    // ---- local-vol grid sigma[j * nK + i], uniform axes
    const float* lv;
    const float2* lv_rows;   // [n_steps + 1] time rows of the fine steps (lv_time_row)
    int lv_nK, lv_nt;
    float lv_K0, lv_inv_dK, lv_t0, lv_inv_dt;
    // ---- Brownian bridge, one row per Sobol dimension j (= bb_precompute step j):
    //      bb[j] = {wl, wr, sd, bits(m)}, bbi[j] = {l, r}
    const float4* bb;
    const int2* bbi;
    float bbw[5][3];    // NOISE_BB_UNI: (wl, wr, sd) of window level u = 0..4
    // ---- PCA: M_pca (fp16, K-major rows = output step) device pointer
    const void* pca;
    // ---- Sobol: pre-scrambled words, replica r at dirs + r * 33 * dstride, word k of dim d at
    //      [k * dstride + d] (k = 32 is the digital shift); dstride >= D (the table may cover more
    //      dimensions than this pass uses, as the book's per-level tables do)
    const uint32_t* dirs;
    int dstride;
    // ---- Philox
    uint32_t seed, stream_base;
    // ---- output: per-item partial sums [n_items][nstat]
    double* partials;
    // ---- parity dump (DumpC only): [R][n_points][D] normals (raw) or increments (bridge)
    float* dump;
    // ---- adjoint: per-node local-vol sensitivities, summed over paths (FP64)
    double* node_out;
    // ---- bounded-wait / error reporting
    int* err;
    // ---- NOISE_DW: increment i of point offset + row at dw_in[i * dw_stride + row]
    const float* dw_in;
    int dw_stride;
};

}  // namespace mcq
