// k_adjoint.cu — pathwise adjoint Greeks on scrambled-Sobol paths (no counterpart in the
// reference, which computes no sensitivities).
//
// For each path (lane) the forward sweep steps S_k -> S_{k+1} = S_k (1 + mu h + sigma_k dW_k),
// keeps the payoff state and checkpoints S every CK steps (16, 32 or 8: an autotuned launch
// variant) in shared memory.  The reverse sweep walks the 32-step Sobol tiles backwards: it
// regenerates the tile's normals (same warp-transposed generator as the pricing pass), recomputes
// each CK-step segment from its checkpoint, and propagates
//     Sbar_k = Sbar_{k+1} dS_{k+1}/dS_k + dP/dS_k,
//     mubar += Sbar_{k+1} S_k h,            sigmabar += Sbar_{k+1} dS_{k+1}/dsigma,
// and, for the grid local-vol model, adds Sbar_{k+1} S_k dW_k w_n to the four bilinear nodes n of
// (S_k, t_k) in an FP32 shared-memory array per CTA (summed per lane over the consecutive steps
// that stay in one grid cell, then added with one native float atomic per node; a path changes
// cell about once a step on the benchmark's grid, and the FP64 shared atomics this replaced were
// the kernel's top stall), whose totals go to the FP64 output once per CTA.  Payoffs are the Lipschitz ones:
// European (discounted), arithmetic Asian and floating-strike lookback (BGK factor constant).
// Per path it yields P, delta = Sbar_0 (plus, for the parametric Dupire model, whose volatility
// (S/S0)^(beta-1) is scaled by S0, the sensitivity through that scale, so that delta is the
// derivative of the price with respect to the model's S0), rho = mubar (+ -T P for the discounted European, the
// drift and the discount sharing the rate) and vega (GBM: d/dsigma; Dupire: d/dsigma0; grid:
// the parallel shift = sum of node vegas; Heston: d/dv0, see k_adjoint_heston).
#include "adjoint.h"
#include "path_kernels.cuh"

namespace mcq {

// Checkpoint interval CK (steps): 16 by default; the autotuner also tries 32 and 8 (a launch
// variant: more or fewer recomputed steps per checkpoint, the same arithmetic and the same bits).
constexpr int kCkVariants[3] = {16, 32, 8};

struct LvEval {
    float sig, dsig;
    int n00;              // node index (j * nK + i) of the lower-left corner
    float w00, w01, w10, w11;
};

// Bilinear sigma(S, t) on the uniform grid exactly as the pricing pass's lv_sigma_row, with dsigma/dS
// and the weights.  The time axis comes from the same per-step rows {j nK (as float bits), b}
// (lv_time_row, path_kernels.cuh), which the CTA forms once in shared memory; the sweeps read them
// instead of clamping, truncating and converting t in each of the three evaluations per step.
__device__ __forceinline__ LvEval lv_eval_row(const KParams& p, float S, float2 row) {
    LvEval e;
    float x = (S - p.lv_K0) * p.lv_inv_dK;
    const bool inside = x > 0.f && x < (float)(p.lv_nK - 1);
    x = fminf(fmaxf(x, 0.f), (float)(p.lv_nK - 1));
    const int i = min((int)x, p.lv_nK - 2);
    const float a = x - (float)i;
    const int jn = __float_as_int(row.x);
    const float b = row.y;
    const float* g = p.lv + jn + i;
    const float s00 = __ldg(g), s01 = __ldg(g + 1), s10 = __ldg(g + p.lv_nK), s11 = __ldg(g + p.lv_nK + 1);
    const float lo = fmaf(a, s01 - s00, s00), hi = fmaf(a, s11 - s10, s10);
    e.sig = fmaf(b, hi - lo, lo);
    e.dsig = inside ? ((1.f - b) * (s01 - s00) + b * (s11 - s10)) * p.lv_inv_dK : 0.f;
    e.n00 = jn + i;
    e.w00 = (1.f - a) * (1.f - b);
    e.w01 = a * (1.f - b);
    e.w10 = (1.f - a) * b;
    e.w11 = a * b;
    return e;
}

// local volatility and its S-derivative / sigma-parameter derivative for the model at step k
// (t = k h; the grid model reads its time row from `trow`)
template <int MOD>
__device__ __forceinline__ float local_sigma(const KParams& p, float S, int k, const float2* trow, float* dsig_dS,
                                             float* dsig_dpar, LvEval* lv) {
    const float t = (float)k * p.h;
    if constexpr (MOD == MOD_GBM) {
        *dsig_dS = 0.f;
        *dsig_dpar = 1.f;
        return p.sigma;
    } else if constexpr (MOD == MOD_DUPIRE) {
        const float sl = p.sigma0 * exp2f(fmaf(p.bm1, log2f(S * p.inv_S0), -p.alpha * t * kLog2e));
        *dsig_dS = sl * p.bm1 / S;
        *dsig_dpar = sl / p.sigma0;
        return sl;
    } else {
        *lv = lv_eval_row(p, S, trow[k]);
        *dsig_dS = lv->dsig;
        *dsig_dpar = 1.f;
        return lv->sig;
    }
}

template <int MOD, int PAY, int CK>
__global__ void __launch_bounds__(kThreads, 2) k_adjoint(const __grid_constant__ KParams p) {
    constexpr int kCk = CK;
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int N = p.n_steps;
    const int n_ck = N / kCk + 1;
    const int per_warp = 1024 + n_ck * 32 + kCk * 32;
    float* nodes = reinterpret_cast<float*>(smem4);               // [n_nodes] FP32, CTA-wide
    const int node_floats = (MOD == MOD_LVGRID) ? ((p.lv_nK * p.lv_nt + 3) & ~3) : 0;
    const int trow_floats = (MOD == MOD_LVGRID) ? ((2 * (N + 1) + 3) & ~3) : 0;
    float2* trow = reinterpret_cast<float2*>(nodes + node_floats);   // [N + 1] time rows (grid model)
    float* wbase = nodes + node_floats + trow_floats + wib * per_warp;
    // each tile's Sobol start word, carried from group to group by the forward sweep and reused
    // as is by the reverse sweep's regeneration of the same tile: slot 32 t + lane, after the warps
    uint32_t* carry = reinterpret_cast<uint32_t*>(nodes + node_floats + trow_floats + kWarpsPerBlock * per_warp) +
                      wib * N;
    float* buf = wbase;               // 32 x 32 transpose tile
    float* ck = wbase + 1024;         // checkpoints [n_ck][32]
    float* seg = ck + n_ck * 32;      // recomputed segment [CK][32]
    if constexpr (MOD == MOD_LVGRID) {
        for (int i = threadIdx.x; i < node_floats; i += blockDim.x) nodes[i] = 0.f;
        for (int k = threadIdx.x; k <= N; k += blockDim.x) trow[k] = lv_time_row(p, k);
        __syncthreads();
    }
    const float h = p.h, sqh = p.sqrt_h, muh = p.mu * p.h;
    const int total_warps = gridDim.x * kWarpsPerBlock;
    const uint64_t gend_all = p.g0 + p.G;
    for (int item = blockIdx.x * kWarpsPerBlock + wib; item < p.n_items; item += total_warps) {
        const int r = item / p.items_per_rep;
        const int j = item - r * p.items_per_rep;
        const uint64_t gb = p.g0 + (uint64_t)j * (uint64_t)p.gpi;
        const uint64_t ge = min(gb + (uint64_t)p.gpi, gend_all);
        const uint32_t* dr = p.dirs + (size_t)r * 33 * (size_t)N;
        Acc<4> acc;
        acc.zero();
        for (uint64_t hg = gb; hg < ge; hg++) {
            const uint64_t n = hg * 32 + (uint64_t)lane;
            const bool valid = n >= p.offset && n < p.offset + p.n_points;
            // ---------------- forward sweep
            float S = p.S0, ts = 0.f, tot = 0.f, comp = 0.f, mn = p.S0;
            int kmin = 0;
            for (int d0 = 0; d0 < N; d0 += 32) {
                sobol_tile(dr, N, d0 + lane, true, hg, p.u_cap, buf, lane, carry + d0 + lane, hg != gb ? 1 : 0);
                __syncwarp();
                // the step loops read this lane's row of the tile from shared memory, four steps
                // per float4 (the swizzled layout makes row reads conflict-free), and stay rolled
                // over the chunks: fully unrolled, the sweeps overflowed the instruction cache
                const float4* row4 = reinterpret_cast<const float4*>(buf + lane * 32);
#pragma unroll 1
                for (int c = 0; c < 8; c++) {
                    const float4 v4 = row4[c ^ (lane & 7)];
                    const float zc[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int i = 4 * c + q;
                        const int k = d0 + i;
                        if ((i & (kCk - 1)) == 0) ck[(k / kCk) * 32 + lane] = S;
                        float dsS, dsP;
                        LvEval lv;
                        const float sig = local_sigma<MOD>(p, S, k, trow, &dsS, &dsP, &lv);
                        S = fmaf(S, fmaf(sig, zc[q] * sqh, muh), S);
                        if constexpr (PAY == PAY_ASIAN) ts += S;
                        if constexpr (PAY == PAY_LOOKBACK) {
                            if (S < mn) { mn = S; kmin = k + 1; }
                        }
                    }
                }
                if constexpr (PAY == PAY_ASIAN) { kadd(tot, comp, ts); ts = 0.f; }
                __syncwarp();
            }
            // payoff and its direct derivatives
            float P, g_all = 0.f, Sbar;
            if constexpr (PAY == PAY_EUR) {
                P = fmaxf(S - p.K, 0.f) * p.disc;
                Sbar = (S > p.K) ? p.disc : 0.f;
            } else if constexpr (PAY == PAY_ASIAN) {
                const float A = (tot - comp) / (float)N;
                P = fmaxf(A - p.K, 0.f);
                g_all = (A > p.K) ? 1.f / (float)N : 0.f;
                Sbar = g_all;
            } else {   // floating-strike lookback
                P = S - mn * p.corr_f;
                Sbar = 1.f + ((kmin == N) ? -p.corr_f : 0.f);
            }
            // ---------------- reverse sweep
            float mubar = 0.f, sigbar = 0.f, s0bar = 0.f;
            // grid local vol: the node sensitivities of consecutive steps in the same cell are
            // summed in registers (FP64) and added to the CTA's node array when the cell changes
            int vcell = -1;
            float v00 = 0.f, v01 = 0.f, v10 = 0.f, v11 = 0.f;
            for (int d0 = N - 32; d0 >= 0; d0 -= 32) {
                sobol_tile(dr, N, d0 + lane, true, hg, p.u_cap, buf, lane, carry + d0 + lane, 2);
                __syncwarp();
                const float4* row4 = reinterpret_cast<const float4*>(buf + lane * 32);
#pragma unroll 1
                for (int s = 32 / kCk - 1; s >= 0; s--) {
                    const int k0 = d0 + s * kCk;
                    float Sr = ck[(k0 / kCk) * 32 + lane];
#pragma unroll 1
                    for (int c = 0; c < kCk / 4; c++) {
                        const float4 v4 = row4[(s * (kCk / 4) + c) ^ (lane & 7)];
                        const float zc[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const int i = 4 * c + q;
                            seg[i * 32 + lane] = Sr;
                            float dsS, dsP;
                            LvEval lv;
                            const float sig = local_sigma<MOD>(p, Sr, k0 + i, trow, &dsS, &dsP, &lv);
                            Sr = fmaf(Sr, fmaf(sig, zc[q] * sqh, muh), Sr);
                        }
                    }
#pragma unroll 1
                    for (int c = kCk / 4 - 1; c >= 0; c--) {
                        const float4 v4 = row4[(s * (kCk / 4) + c) ^ (lane & 7)];
                        const float zc[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                        for (int q = 3; q >= 0; q--) {
                            const int i = 4 * c + q;
                            const int k = k0 + i;
                            const float Sk = seg[i * 32 + lane];
                            const float dw = zc[q] * sqh;
                            float dsS, dsP;
                            LvEval lv;
                            const float sig = local_sigma<MOD>(p, Sk, k, trow, &dsS, &dsP, &lv);
                            mubar = fmaf(Sbar, Sk * h, mubar);
                            const float sens = Sbar * Sk * dw;     // dP/dsigma_k through this step
                            sigbar = fmaf(sens, dsP, sigbar);
                            // the parametric Dupire volatility is scaled by the model's S0 itself:
                            // d sigma_k / d S0 = -(beta - 1) sigma_k / S0 enters the delta
                            if constexpr (MOD == MOD_DUPIRE) s0bar = fmaf(sens, -p.bm1 * sig * p.inv_S0, s0bar);
                            if constexpr (MOD == MOD_LVGRID) {
                                if (valid && sens != 0.f) {
                                    if (lv.n00 != vcell) {
                                        if (vcell >= 0) {
                                            atomicAdd(&nodes[vcell], v00);
                                            atomicAdd(&nodes[vcell + 1], v01);
                                            atomicAdd(&nodes[vcell + p.lv_nK], v10);
                                            atomicAdd(&nodes[vcell + p.lv_nK + 1], v11);
                                        }
                                        vcell = lv.n00;
                                        v00 = v01 = v10 = v11 = 0.f;
                                    }
                                    v00 = fmaf(sens, lv.w00, v00);
                                    v01 = fmaf(sens, lv.w01, v01);
                                    v10 = fmaf(sens, lv.w10, v10);
                                    v11 = fmaf(sens, lv.w11, v11);
                                }
                            }
                            const float dS1 = 1.f + muh + sig * dw + Sk * dw * dsS;
                            float direct = 0.f;
                            if constexpr (PAY == PAY_ASIAN) direct = (k >= 1) ? g_all : 0.f;
                            if constexpr (PAY == PAY_LOOKBACK) direct = (k == kmin) ? -p.corr_f : 0.f;
                            Sbar = fmaf(Sbar, dS1, direct);
                        }
                    }
                }
                __syncwarp();
            }
            if constexpr (MOD == MOD_LVGRID) {
                if (vcell >= 0) {
                    atomicAdd(&nodes[vcell], v00);
                    atomicAdd(&nodes[vcell + 1], v01);
                    atomicAdd(&nodes[vcell + p.lv_nK], v10);
                    atomicAdd(&nodes[vcell + p.lv_nK + 1], v11);
                }
            }
            float rho = mubar;
            if constexpr (PAY == PAY_EUR) rho -= p.pay_T * P;
            float y[4] = {P, Sbar + s0bar, rho, sigbar};
            if (valid) acc.add(y);
        }
        acc.flush(p.partials + (size_t)item * 4, lane);
    }
    if constexpr (MOD == MOD_LVGRID) {
        __syncthreads();
        for (int i = threadIdx.x; i < p.lv_nK * p.lv_nt; i += blockDim.x)
            if (nodes[i] != 0.f) atomicAdd(p.node_out + i, (double)nodes[i]);
    }
}

// Heston (two normals per step: dims 2k for the price, 2k + 1 for the variance, correlated by the
// Cholesky row (L10, L11)), the pricing pass's Euler step with full truncation in the square
// root (and, with MCQ_FLAG_HESTON_MILSTEIN, the Milstein term, which does not depend on V):
//     S' = S + S (mu h + sqrt(V+) dW1),   V' = theta + e^{-kappa h} (V - theta) + xi sqrt(V+) dW2.
// The reverse sweep carries (Sbar, Vbar):
//     Sbar_k = Sbar_{k+1} (1 + mu h + sqrt(V+) dW1) + dP/dS_k,
//     Vbar_k = Sbar_{k+1} S_k dW1 s'(V_k) + Vbar_{k+1} (e^{-kappa h} + xi dW2 s'(V_k)),
// with s'(V) = 1 / (2 sqrt V) for V > 0 and the subgradient 0 where the truncation is active.
// Outputs per path: P, delta = Sbar_0, rho = mubar (- T P for the discounted European) and
// vega = Vbar_0 = dP/dv0.  A 32-dimension Sobol tile is 16 steps, which is also the checkpoint
// interval: (S, V) are kept at every tile boundary.
__device__ __forceinline__ void heston_adj_step(const KParams& p, float& S, float& V, float dw1, float dw2,
                                                float muh) {
    const float sq = sqrtf(fmaxf(V, 0.f));
    // the pricing pass's operations (Leg::step): one rounding against S and one against V
    S = fmaf(S, fmaf(sq, dw1, muh), S);
    float inc = fmaf(p.xi * sq, dw2, p.om_f * (p.theta - V));
    inc = (p.mil != 0.f) ? fmaf(p.mil, fmaf(dw2, dw2, -p.h), inc) : inc;
    V = V + inc;
}

template <int PAY>
__global__ void __launch_bounds__(kThreads, 1) k_adjoint_heston(const __grid_constant__ KParams p) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int N = p.n_steps, D = 2 * N, n_tiles = D / 32;
    const int per_warp = 1024 + (n_tiles + 1) * 64 + 16 * 64;
    float* wbase = reinterpret_cast<float*>(smem4) + wib * per_warp;
    float* buf = wbase;                       // 32 x 32 transpose tile
    float* ckS = wbase + 1024;                // (S, V) at every tile boundary [n_tiles + 1][32]
    float* ckV = ckS + (n_tiles + 1) * 32;
    float* segS = ckV + (n_tiles + 1) * 32;   // the recomputed tile [16][32]
    float* segV = segS + 16 * 32;
    const float h = p.h, sqh = p.sqrt_h, muh = p.mu * p.h;
    const int total_warps = gridDim.x * kWarpsPerBlock;
    const uint64_t gend_all = p.g0 + p.G;
    for (int item = blockIdx.x * kWarpsPerBlock + wib; item < p.n_items; item += total_warps) {
        const int r = item / p.items_per_rep;
        const int j = item - r * p.items_per_rep;
        const uint64_t gb = p.g0 + (uint64_t)j * (uint64_t)p.gpi;
        const uint64_t ge = min(gb + (uint64_t)p.gpi, gend_all);
        const uint32_t* dr = p.dirs + (size_t)r * 33 * (size_t)D;
        Acc<4> acc;
        acc.zero();
        for (uint64_t hg = gb; hg < ge; hg++) {
            const uint64_t n = hg * 32 + (uint64_t)lane;
            const bool valid = n >= p.offset && n < p.offset + p.n_points;
            // ---------------- forward sweep
            float S = p.S0, V = p.v0, ts = 0.f, tot = 0.f, comp = 0.f, mn = p.S0;
            int kmin = 0;
            for (int t = 0; t < n_tiles; t++) {
                ckS[t * 32 + lane] = S;
                ckV[t * 32 + lane] = V;
                sobol_tile(dr, D, t * 32 + lane, true, hg, p.u_cap, buf, lane);
                __syncwarp();
                float z[32];
                read_row(buf, lane, z);
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const float z1 = z[2 * i], z2 = z[2 * i + 1];
                    heston_adj_step(p, S, V, z1 * sqh, fmaf(p.L10, z1, p.L11 * z2) * sqh, muh);
                    if constexpr (PAY == PAY_ASIAN) ts += S;
                    if constexpr (PAY == PAY_LOOKBACK) {
                        if (S < mn) { mn = S; kmin = t * 16 + i + 1; }
                    }
                }
                if constexpr (PAY == PAY_ASIAN) { kadd(tot, comp, ts); ts = 0.f; }
            }
            float P, g_all = 0.f, Sbar;
            if constexpr (PAY == PAY_EUR) {
                P = fmaxf(S - p.K, 0.f) * p.disc;
                Sbar = (S > p.K) ? p.disc : 0.f;
            } else if constexpr (PAY == PAY_ASIAN) {
                const float A = (tot - comp) / (float)N;
                P = fmaxf(A - p.K, 0.f);
                g_all = (A > p.K) ? 1.f / (float)N : 0.f;
                Sbar = g_all;
            } else {   // floating-strike lookback
                P = S - mn * p.corr_f;
                Sbar = 1.f + ((kmin == N) ? -p.corr_f : 0.f);
            }
            // ---------------- reverse sweep
            float mubar = 0.f, Vbar = 0.f;
            for (int t = n_tiles - 1; t >= 0; t--) {
                sobol_tile(dr, D, t * 32 + lane, true, hg, p.u_cap, buf, lane);
                __syncwarp();
                float z[32];
                read_row(buf, lane, z);
                __syncwarp();
                float Sr = ckS[t * 32 + lane], Vr = ckV[t * 32 + lane];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    segS[i * 32 + lane] = Sr;
                    segV[i * 32 + lane] = Vr;
                    const float z1 = z[2 * i], z2 = z[2 * i + 1];
                    heston_adj_step(p, Sr, Vr, z1 * sqh, fmaf(p.L10, z1, p.L11 * z2) * sqh, muh);
                }
#pragma unroll
                for (int i = 15; i >= 0; i--) {
                    const int k = t * 16 + i;
                    const float Sk = segS[i * 32 + lane], Vk = segV[i * 32 + lane];
                    const float z1 = z[2 * i], z2 = z[2 * i + 1];
                    const float dw1 = z1 * sqh, dw2 = fmaf(p.L10, z1, p.L11 * z2) * sqh;
                    const float sq = sqrtf(fmaxf(Vk, 0.f));
                    const float dsq = (Vk > 0.f) ? 0.5f / sq : 0.f;
                    mubar = fmaf(Sbar, Sk * h, mubar);
                    const float nV = fmaf(Sbar, Sk * dw1 * dsq, Vbar * fmaf(p.xi * dw2, dsq, 1.f - p.om_f));
                    float direct = 0.f;
                    if constexpr (PAY == PAY_ASIAN) direct = (k >= 1) ? g_all : 0.f;
                    if constexpr (PAY == PAY_LOOKBACK) direct = (k == kmin) ? -p.corr_f : 0.f;
                    Sbar = fmaf(Sbar, 1.f + muh + sq * dw1, direct);
                    Vbar = nV;
                }
            }
            float rho = mubar;
            if constexpr (PAY == PAY_EUR) rho -= p.pay_T * P;
            float y[4] = {P, Sbar, rho, Vbar};
            if (valid) acc.add(y);
        }
        acc.flush(p.partials + (size_t)item * 4, lane);
    }
}

template <int MOD, int CK>
static const void* adj_payoff(int pay) {
    switch (pay) {
        case PAY_EUR: return (const void*)&k_adjoint<MOD, PAY_EUR, CK>;
        case PAY_ASIAN: return (const void*)&k_adjoint<MOD, PAY_ASIAN, CK>;
        case PAY_LOOKBACK: return (const void*)&k_adjoint<MOD, PAY_LOOKBACK, CK>;
        default: return nullptr;
    }
}

template <int MOD>
static const void* adj_ck(int pay, int variant) {
    switch (variant) {
        case 1: return adj_payoff<MOD, kCkVariants[1]>(pay);
        case 2: return adj_payoff<MOD, kCkVariants[2]>(pay);
        default: return adj_payoff<MOD, kCkVariants[0]>(pay);
    }
}

int adjoint_variants(int model) { return model == MOD_HESTON ? 1 : 3; }

const void* lookup_adjoint(int model, int payoff, int variant) {
    switch (model) {
        case MOD_GBM: return adj_ck<MOD_GBM>(payoff, variant);
        case MOD_DUPIRE: return adj_ck<MOD_DUPIRE>(payoff, variant);
        case MOD_LVGRID: return adj_ck<MOD_LVGRID>(payoff, variant);
        case MOD_HESTON:
            switch (payoff) {
                case PAY_EUR: return (const void*)&k_adjoint_heston<PAY_EUR>;
                case PAY_ASIAN: return (const void*)&k_adjoint_heston<PAY_ASIAN>;
                case PAY_LOOKBACK: return (const void*)&k_adjoint_heston<PAY_LOOKBACK>;
                default: return nullptr;
            }
        default: return nullptr;
    }
}

size_t adjoint_smem_bytes(int model, int n_steps, int n_nodes, int variant) {
    if (model == MOD_HESTON) {
        const int n_tiles = 2 * n_steps / 32;
        return (size_t)kWarpsPerBlock * (1024 + (n_tiles + 1) * 64 + 16 * 64) * sizeof(float);
    }
    const int ck = kCkVariants[(variant >= 0 && variant < 3) ? variant : 0];
    const int n_ck = n_steps / ck + 1;
    const size_t per_warp = (size_t)(1024 + n_ck * 32 + ck * 32) * sizeof(float);
    const size_t trow = (model == MOD_LVGRID) ? (size_t)((2 * (n_steps + 1) + 3) & ~3) * sizeof(float) : 0;
    const size_t carry = (size_t)kWarpsPerBlock * n_steps * sizeof(uint32_t);   // start-word slots
    return (size_t)((n_nodes + 3) & ~3) * sizeof(float) + trow + kWarpsPerBlock * per_warp + carry;
}

}  // namespace mcq
