// path_kernels.cuh — the fused path kernel for sm_100a.
//
// One launch prices R replicas x n_points paths end to end: point generation (scrambled
// Sobol or Philox), noise transform (raw, Brownian bridge), Euler stepping of the model,
// running payoff accumulator, payoff / control-variate / importance-sampling weights,
// Kahan accumulation per lane and a warp-shuffle reduction per work item.  No path array
// is ever written to HBM; the only global writes are one partial-sum record per item.
//
// This fuses what the reference does in up to five passes over a D x N array in HBM:
//   kernel_gen_hh_scrambled_sobol_normal / curandGenerateNormal   (methods_cuda.cu:799-825)
//   kernel_scale / kernel_bb_transform                             (:561-594, :714-718)
//   kernel_mc / kernel_mlmc / kernel_gbm_asian_cv / kernel_dupire_gbm_cv / kernel_is_gbm
//   with CUB_REDUCE2/4 + atomicAdd                                 (:359-381, :414-707)
//
// Work layout.  Points are taken in aligned groups of 32 consecutive indices, one group per
// warp at a time (lane i owns point 32h + i).  A work item is a run of `gpi` groups of one
// replica; warps take items round-robin.  Item boundaries depend only on the problem size, so
// the result is bit-reproducible run to run.
//
// Sobol generation (warp-transposed).  For a tile of 32 dimensions, lane j owns dimension
// d0 + j and produces its scrambled integers for all 32 points of the group by gray-code
// recurrence: x(32h) = shift ^ XOR_{k in gray(h)} Lv[5+k] ^ [h odd] Lv[4], then
// x(32h+i+1) = x(32h+i) ^ Lv[ctz(i+1)].  Lv are the direction words already multiplied by the
// replica's Hong–Hickernell matrix (linearity of the scramble over F2), so each point costs
// one XOR instead of 32 splitmix32 rows + 32 popcounts (hh_scramble, methods_cuda.cu:781-795).
// The normals go through a 32x32 XOR-swizzled shared-memory transpose and come back one row
// (one path) per lane.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>
#include <cuda_fp16.h>
#include "kparams.h"

namespace mcq {

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kTwoPow32Inv = 2.3283064365386963e-10f;   // 2^-32
constexpr float kTwoPow24Inv = 5.9604644775390625e-08f;   // 2^-24

// Direction word of the gray-code step from point i to point i + 1 inside a block of eight
// (i = 0..6: word ctz(i + 1) = 0, 1, 0, 2, 0, 1, 0), written as bit tests of i so that an unrolled
// i folds to one XOR operand.  (A recursive constexpr ctz called with the loop index is not
// folded by the device compiler: it left ~10 integer and branch instructions per normal.)
__device__ __forceinline__ uint32_t gray_word8(int i, uint32_t L0, uint32_t L1, uint32_t L2) {
    return (i & 1) == 0 ? L0 : ((i & 2) ? L2 : L1);
}

// ------------------------------------------------------------------ hashing / scrambling

// splitmix32 (methods_cuda.cu:753-759).
__host__ __device__ __forceinline__ uint32_t splitmix32(uint32_t x) {
    x += 0x9E3779B9u;
    x = (x ^ (x >> 16)) * 0x21F0AAADu;
    x = (x ^ (x >> 15)) * 0x735A2D97u;
    return x ^ (x >> 15);
}

// Hong–Hickernell lower-triangular F2 matrix applied to v, row k MSB-first, without the
// digital shift (the linear part of hh_scramble, methods_cuda.cu:781-795).
__device__ __forceinline__ uint32_t hh_linear(uint32_t v, uint32_t base) {
    uint32_t out = 0;
#pragma unroll
    for (int k = 0; k < 32; k++) {
        uint32_t seed = splitmix32(base ^ (uint32_t)k);
        uint32_t mask = (k == 0) ? 0u : (0xFFFFFFFFu << (32 - k));
        uint32_t row = (1u << (31 - k)) | (seed & mask);
        out |= ((uint32_t)__popc(row & v) & 1u) << (31 - k);
    }
    return out;
}

// u = ((float)s + 1) * 2^-32 as in methods_cuda.cu:823; u_cap is 1.0f in reference-compat
// mode (u may be 1 -> +inf) and 1 - 2^-24 otherwise.
// ((float)x + 1) * 2^-32 == fma((float)x, 2^-32, 2^-32) bit for bit: scaling by a power of two
// is exact, so both round the same real number once.
__device__ __forceinline__ float sobol_normal(uint32_t x, float u_cap) {
    const float u = fmaf((float)x, kTwoPow32Inv, kTwoPow32Inv);
    return normcdfinvf(fminf(u, u_cap));
}

// ------------------------------------------------------------------ transpose buffer

// 32 x 32 floats per warp, 16-byte chunks XOR-swizzled by row so that column writes
// (lane = column) and float4 row reads (lane = row) are both bank-conflict free.
__device__ __forceinline__ int swz(int row, int col) {
    return row * 32 + ((((col >> 2) ^ (row & 7)) << 2) | (col & 3));
}

__device__ __forceinline__ void read_row(const float* buf, int lane, float (&z)[32]) {
    const float4* b4 = reinterpret_cast<const float4*>(buf + lane * 32);
#pragma unroll
    for (int c = 0; c < 8; c++) {
        float4 v = b4[c ^ (lane & 7)];
        z[4 * c + 0] = v.x; z[4 * c + 1] = v.y; z[4 * c + 2] = v.z; z[4 * c + 3] = v.w;
    }
}

// Lane owns dimension `dim` of replica table `dr` (words [k * D + dim]); writes the normals of
// points 32h .. 32h+31 into column `lane` of the transpose buffer.
//
// The start word x(32h) = shift ^ XOR of v_k over the set bits k of gray(32h), and
// gray(32h) = gray(h) << 5 | (h & 1) << 4, so a tile walks popcount(gray(h)) words from the
// digital shift.  A caller that generates the same dimension for groups h - 1, h, h + 1, ... in
// order keeps the start word of each tile in `slot` (shared memory) and passes cont = 1 from the
// second group on: x(32h) = x(32(h - 1)) ^ v_4 ^ v_{5 + ctz(h)}, two words instead of the walk and
// its chain of dependent loads (the same word, so the same normals).  cont = 2: the slot already
// holds x(32h) (a tile generated again for the same group, as the adjoint's reverse sweep does).
//
// The 32 points run as four blocks of eight: inside a block the gray-code step is fixed (word
// ctz(i + 1), gray_word8), between blocks (points 8, 16, 24) it XORs word 3 + ctz(b + 1).  UNR
// blocks are unrolled at a time (1, 2 or 4): a larger unroll drops the loop's overhead but
// multiplies the inlined inverse-normal code the instruction cache must hold; the fused pass
// families are compiled with more than one and the autotuner picks (the same normals).
__device__ __forceinline__ void sobol_block8(uint32_t& x, int b, uint32_t L0, uint32_t L1, uint32_t L2,
                                             uint32_t L3, uint32_t L4, float u_cap, float* buf, int lane) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
        buf[swz(8 * b + i, lane)] = sobol_normal(x, u_cap);
        if (i < 7) x ^= gray_word8(i, L0, L1, L2);
        else if (b < 3) x ^= (b == 1) ? L4 : L3;
    }
}

template <int UNR = 1>
__device__ __forceinline__ void sobol_tile(const uint32_t* __restrict__ dr, int D, int dim,
                                           bool active, uint64_t h, float u_cap, float* buf,
                                           int lane, uint32_t* slot = nullptr, int cont = 0) {
    static_assert(UNR == 1 || UNR == 2 || UNR == 4, "blocks unrolled: 1, 2 or 4");
    if (!active) return;
    const uint32_t* col = dr + dim;
    const uint32_t L0 = __ldg(col), L1 = __ldg(col + D), L2 = __ldg(col + 2 * D),
                   L3 = __ldg(col + 3 * D), L4 = __ldg(col + 4 * D);
    uint32_t x;
    if (slot != nullptr && cont == 2) {
        x = *slot;
    } else if (slot != nullptr && cont) {
        x = *slot ^ L4 ^ __ldg(col + (4 + __ffsll((long long)h)) * D);
    } else {
        x = __ldg(col + 32 * D);
        if (h & 1) x ^= L4;
        uint32_t g = (uint32_t)(h ^ (h >> 1));
        while (g) {
            const int k = __ffs(g) - 1;
            x ^= __ldg(col + (5 + k) * D);
            g &= g - 1;
        }
    }
    if (slot != nullptr) *slot = x;
    if constexpr (UNR == 4) {
#pragma unroll
        for (int b = 0; b < 4; b++) sobol_block8(x, b, L0, L1, L2, L3, L4, u_cap, buf, lane);
    } else if constexpr (UNR == 2) {
#pragma unroll 2
        for (int b = 0; b < 4; b++) sobol_block8(x, b, L0, L1, L2, L3, L4, u_cap, buf, lane);
    } else {
#pragma unroll 1
        for (int b = 0; b < 4; b++) sobol_block8(x, b, L0, L1, L2, L3, L4, u_cap, buf, lane);
    }
}

// ------------------------------------------------------------------ Philox4x32-10

__device__ __forceinline__ uint4 philox10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r) { k.x += 0x9E3779B9u; k.y += 0xBB67AE85u; }
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, float& z0, float& z1) {
    const float u1 = ((float)(a >> 8) + 0.5f) * kTwoPow24Inv;
    const float u2 = ((float)(b >> 8) + 0.5f) * kTwoPow24Inv;
    const float rr = sqrtf(-2.0f * logf(u1));
    float s, c;
    sincospif(2.0f * u2, &s, &c);
    z0 = rr * s;
    z1 = rr * c;
}

// Normals 32t .. 32t+31 of path `path` on stream `stream` (block b = dims 4b..4b+3).
__device__ __forceinline__ void philox_tile(uint32_t seed, uint32_t stream, uint64_t path, int t,
                                            float (&z)[32]) {
    const uint2 key = make_uint2(seed, 0x6D637121u);
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const uint4 o = philox10(make_uint4((uint32_t)(8 * t + q), (uint32_t)path,
                                            (uint32_t)(path >> 32), stream), key);
        box_muller(o.x, o.y, z[4 * q], z[4 * q + 1]);
        box_muller(o.z, o.w, z[4 * q + 2], z[4 * q + 3]);
    }
}

// ------------------------------------------------------------------ accumulation

__device__ __forceinline__ void kadd(float& s, float& c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

template <int NST>
struct Acc {
    float s[NST], c[NST];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < NST; i++) s[i] = c[i] = 0.f;
    }
    __device__ __forceinline__ void add(const float (&y)[NST]) {
#pragma unroll
        for (int i = 0; i < NST; i++) kadd(s[i], c[i], y[i]);
    }
    // Warp total in FP64 (fixed shuffle order), lane 0 stores the item record.
    __device__ __forceinline__ void flush(double* out, int lane) {
#pragma unroll
        for (int i = 0; i < NST; i++) {
            double v = (double)s[i] - (double)c[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) out[i] = v;
        }
    }
};

// Accumulator for consumers with many statistics: each group's 32 values are reduced in FP32
// by shuffles and lane 0 adds the group total to an FP64 record in the warp's shared memory.
template <int NST>
struct AccWarp {
    double* rec;
    __device__ __forceinline__ void bind(double* r, int lane) {
        rec = r;
        if (lane < NST) rec[lane] = 0.0;
        __syncwarp();
    }
    __device__ __forceinline__ void add(const float (&y)[NST], bool valid, int lane) {
#pragma unroll
        for (int i = 0; i < NST; i++) {
            float v = valid ? y[i] : 0.f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) rec[i] += (double)v;
        }
    }
    __device__ __forceinline__ void flush(double* out, int lane) {
        __syncwarp();
        if (lane < NST) out[lane] = rec[lane];
        __syncwarp();
    }
};

// ------------------------------------------------------------------ models and payoffs

// Grid local volatility, bilinear in (S, t) on the uniform axes.  Every path of a step k shares
// t = k h, so the time axis comes from a per-step row {j nK (as float bits), b} that the engine forms
// once per pass (k_lv_rows) with these expressions; the paths then read it instead of clamping,
// truncating and converting t at every step (the same values, bit for bit).
__device__ __forceinline__ float2 lv_time_row(const KParams& p, int k) {
    const float t = (float)k * p.h;
    float y = (t - p.lv_t0) * p.lv_inv_dt;
    y = fminf(fmaxf(y, 0.f), (float)(p.lv_nt - 1));
    const int j = min((int)y, p.lv_nt - 2);
    return make_float2(__int_as_float(j * p.lv_nK), y - (float)j);
}

__device__ __forceinline__ float lv_sigma_row(const KParams& p, float S, float2 row) {
    float x = (S - p.lv_K0) * p.lv_inv_dK;
    x = fminf(fmaxf(x, 0.f), (float)(p.lv_nK - 1));
    const int i = min((int)x, p.lv_nK - 2);
    const float a = x - (float)i;
    const float b = row.y;
    const float* g = p.lv + __float_as_int(row.x) + i;
    const float s00 = __ldg(g), s01 = __ldg(g + 1), s10 = __ldg(g + p.lv_nK),
                s11 = __ldg(g + p.lv_nK + 1);
    const float lo = fmaf(a, s01 - s00, s00), hi = fmaf(a, s11 - s10, s10);
    return fmaf(b, hi - lo, lo);
}

// sqrt(V+) of the Heston step with the hardware's approximate square root (`sqrt.approx.f32`,
// relative error about 2^-23, exact at 0 and +inf) instead of the correctly rounded one, whose
// refinement and special-case branch cost 9 % of a coupled Heston level pass.  The error scales
// the diffusion coefficient of S and V by 1 +- 1e-7 and does not enter any drift, so it biases
// neither the level means nor their differences.
__device__ __forceinline__ float sqrt_approx(float v) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(v));
    return r;
}

// Parametric Dupire local volatility sigma0 e^{-alpha t} (S/S0)^(beta - 1) = sigma0 2^{(beta - 1) log2(S/S0)
// - alpha t log2(e)}, x = S/S0, with the hardware's approximate base-2 logarithm and exponential
// (`lg2.approx.f32`, `ex2.approx.f32`: errors about 2^-22, the same special values: log2 of 0 is
// -inf, of a negative x NaN, 2^-inf = 0).  As with the Heston square root, the error scales the
// volatility (1 +- 1e-6), which multiplies only the mean-zero increment: it biases no drift.
__device__ __forceinline__ float dupire_vol(const KParams& p, float x, float t) {
    float l, e;
    asm("lg2.approx.f32 %0, %1;" : "=f"(l) : "f"(x));
    const float a = fmaf(p.bm1, l, -p.alpha * t * kLog2e);
    asm("ex2.approx.f32 %0, %1;" : "=f"(e) : "f"(a));
    return p.sigma0 * e;
}

template <int PAY>
__host__ __device__ constexpr bool path_dep() {
    return PAY == PAY_ASIAN || PAY == PAY_GEOM || PAY == PAY_LOOKBACK || PAY == PAY_UPOUT ||
           PAY == PAY_DOWNOUT;
}

// One discretisation of one single-asset path (d_euler_gbm / d_euler_heston / d_euler_dupire
// and d_running_* / d_apply_bgk / d_payoff, methods_cuda.cu:270-352).  The Euler update is
// S + S (mu h + vol dW), two FMAs; the reference's S + mu S h + vol S dW differs only in
// rounding.  (Folding the drift into a constant 1 + mu h would round that constant once and
// repeat the same relative error on every step: a systematic drift bias of up to 3e-4 of
// mu h per step that does not cancel between the fine and coarse paths of an MLMC level.)
template <int MOD, int PAY>
struct Leg {
    // running accumulator: sums (Asian, geometric) keep a plain partial `tp` over at most 32
    // steps that flush() folds into the Kahan pair (r0, r1); extrema live in r0
    float S, V, r0, r1, tp;
    static constexpr bool SUM = (PAY == PAY_ASIAN || PAY == PAY_GEOM);
    __device__ __forceinline__ void init(const KParams& p) {
        S = p.S0; V = p.v0; r1 = 0.f; tp = 0.f;
        r0 = (PAY == PAY_LOOKBACK || PAY == PAY_DOWNOUT) ? p.S0 : 0.f;
    }
    __device__ __forceinline__ void flush() {
        if constexpr (SUM) { kadd(r0, r1, tp); tp = 0.f; }
    }
    __device__ __forceinline__ void update() {
        if constexpr (PAY == PAY_ASIAN) tp += S;
        else if constexpr (PAY == PAY_GEOM) tp += logf(S);
        else if constexpr (PAY == PAY_LOOKBACK || PAY == PAY_DOWNOUT) r0 = fminf(r0, S);
        else if constexpr (PAY == PAY_UPOUT) r0 = fmaxf(r0, S);
    }
    // update() when `on`, as selects rather than a branch per step (the same values)
    __device__ __forceinline__ void update_if(bool on) {
        if constexpr (PAY == PAY_ASIAN) tp += on ? S : 0.f;
        else if constexpr (PAY == PAY_GEOM) { if (on) tp += logf(S); }
        else if constexpr (PAY == PAY_LOOKBACK || PAY == PAY_DOWNOUT) r0 = on ? fminf(r0, S) : r0;
        else if constexpr (PAY == PAY_UPOUT) r0 = on ? fmaxf(r0, S) : r0;
    }
    // t = ks h is step ks's time (the grid local-vol model reads its time row ks instead)
    template <bool RUN>
    __device__ __forceinline__ void step(const KParams& p, float dw1, float dw2, float t,
                                         float muh, float omk, float hstep, int ks) {
        if constexpr (MOD == MOD_GBM) {
            S = fmaf(S, fmaf(p.sigma, dw1, muh), S);
        } else if constexpr (MOD == MOD_DUPIRE) {
            const float sl = dupire_vol(p, S * p.inv_S0, t);
            S = fmaf(S, fmaf(sl, dw1, muh), S);
        } else if constexpr (MOD == MOD_LVGRID) {
            const float sl = lv_sigma_row(p, S, __ldg(p.lv_rows + ks));
            S = fmaf(S, fmaf(sl, dw1, muh), S);
        } else if constexpr (MOD == MOD_HESTON) {
            // S + S (mu h + sqrt(V+) dW1): the drift joins the random increment before the one
            // rounding against S (S + mu h S rounded on its own would quantise the drift of a fine
            // step, a few ulps of S, the same way at every step: a bias at 2^18 steps)
            const float sq = sqrt_approx(fmaxf(V, 0.f));
            const float Sp = S;
            S = fmaf(S, fmaf(sq, dw1, muh), S);
            if (p.flags & MCQ_FLAG_COMPAT_U_INF_CODE) {
                // reference-compat: a path that went infinite (u = 1 point) and whose variance
                // truncates to 0 becomes NaN through the reference's product sqrt(V+) S (:280)
                const float t0 = sq * Sp;
                if (t0 != t0) S = t0;
            }
            // V + (1 - e^{-kappa h}) (theta - V) + xi sqrt(V+) dW2 (+ xi^2/4 (dW2^2 - h) with the
            // Milstein flag): the reference's exact-mean Euler step (:282-283) with 1 - e^{-kappa h}
            // at full relative precision, and every term summed into one increment before the one
            // rounding against V.  A deterministic term rounded against V on its own (V - xi^2 h / 4,
            // or V + (1 - e^{-kappa h})(theta - V)) leaves the same fraction of an ulp every fine
            // step: at 2^18 steps a drift of V of ~0.5 % that the level differences do not cancel.
            // The Milstein choice is a select on the parameter block (no branch per step); without
            // the flag the term is not formed at all, so an infinite normal of the reference-compat
            // u = 1 point leaves V = +inf as the reference's step does, not 0 * inf = NaN.
            float inc = fmaf(p.xi * sq, dw2, omk * (p.theta - V));
            inc = (p.mil != 0.f) ? fmaf(p.mil, fmaf(dw2, dw2, -hstep), inc) : inc;
            V = V + inc;
        }
        if constexpr (RUN && path_dep<PAY>()) update();
    }
    // GBM step from a raw normal: S + S (mu h + (sigma sqrt h) z)
    __device__ __forceinline__ void step_gbm_z(float z, float sig_sqh, float muh) {
        S = fmaf(S, fmaf(sig_sqh, z, muh), S);
        if constexpr (path_dep<PAY>()) update();
    }
    __device__ __forceinline__ float payoff(const KParams& p, int n, float corr) const {
        if constexpr (PAY == PAY_EUR || PAY == PAY_BASKET) return fmaxf(S - p.K, 0.f) * p.disc;
        else if constexpr (PAY == PAY_ASIAN) return fmaxf((r0 - r1) / (float)n - p.K, 0.f);
        else if constexpr (PAY == PAY_GEOM) return fmaxf(expf((r0 - r1) / (float)n) - p.K, 0.f);
        else if constexpr (PAY == PAY_LOOKBACK) return S - r0 * corr;
        else if constexpr (PAY == PAY_UPOUT) return (r0 / corr >= p.B) ? 0.f : fmaxf(S - p.K, 0.f) * p.disc;
        else return (r0 * corr <= p.B) ? 0.f : fmaxf(S - p.K, 0.f) * p.disc;   // PAY_DOWNOUT
    }
};

// ------------------------------------------------------------------ path consumers
// A consumer takes the normals of its path in Sobol-dimension order (raw mode, tile by tile)
// or the time-ordered increments (bridge mode) and produces the estimator's statistics.

// Single-level / coupled fine-coarse path (kernel_mc, kernel_mlmc).
template <int MOD, int PAY, bool COUPLED>
struct PathC {
    // the grid local-vol time rows are those of the fine steps (a coarse leg would need its own)
    static_assert(!(COUPLED && MOD == MOD_LVGRID), "no coupled grid local-vol pass");
    static constexpr int NST = COUPLED ? 4 : 2;
    __device__ __forceinline__ void bind(int, uint64_t) {}
    static constexpr bool HES = (MOD == MOD_HESTON);
    Leg<MOD, PAY> f, c;
    float a1, a2, muh_f, muh_c;   // mu h of the fine and coarse steps
    int k, m, ck;
    bool run_upd;
    __device__ __forceinline__ void init(const KParams& p) {
        f.init(p);
        muh_f = p.mu * p.h;
        k = 0;
        run_upd = !(HES && COUPLED && (p.flags & 2));
        if constexpr (COUPLED) { c.init(p); a1 = a2 = 0.f; m = 0; ck = 0; muh_c = p.mu * p.hc; }
    }
    // one fine step and, coupled, its increments summed for the coarse step
    __device__ __forceinline__ void fine_dw(const KParams& p, float dw1, float dw2) {
        const float t = (float)k * p.h;
        if constexpr (HES && COUPLED) {   // run_upd is a runtime flag only here
            f.template step<false>(p, dw1, dw2, t, muh_f, p.om_f, p.h, k);
            if constexpr (path_dep<PAY>()) f.update_if(run_upd);
        } else {
            f.template step<true>(p, dw1, dw2, t, muh_f, p.om_f, p.h, k);
        }
        k++;
        if constexpr (COUPLED) {
            a1 += dw1;
            if constexpr (HES) a2 += dw2;
        }
    }
    // the coarse step on the last M fine increments
    __device__ __forceinline__ void coarse_now(const KParams& p) {
        const float tc = (float)ck * p.hc;
        if constexpr (HES) {
            c.template step<false>(p, a1, a2, tc, muh_c, p.om_c, p.hc, ck);
            if constexpr (path_dep<PAY>()) c.update_if(run_upd);
        } else {
            c.template step<true>(p, a1, a2, tc, muh_c, p.om_c, p.hc, ck);
        }
        a1 = a2 = 0.f; ck++;
    }
    __device__ __forceinline__ void step_dw(const KParams& p, float dw1, float dw2) {
        fine_dw(p, dw1, dw2);
        if constexpr (COUPLED) {
            if (++m == p.M) {
                coarse_now(p);
                m = 0;
            }
        }
    }
    // A full tile of a coupled pair with M = MM fine steps per coarse step, entered with no fine
    // step pending (m = 0, which holds at every tile boundary when M divides the tile's steps): the
    // coarse steps fall on compile-time positions instead of a counter test per fine step (the same
    // steps in the same order, so the same bits).
    template <int MM>
    __device__ __forceinline__ void tile_mm(const KParams& p, const float (&z)[32]) {
#pragma unroll
        for (int i = 0; i < 32; i++) {
            fine_dw(p, z[i] * p.sqrt_h, 0.f);
            if ((i % MM) == MM - 1) coarse_now(p);
        }
    }
    template <int MM>
    __device__ __forceinline__ void tile_hes_mm(const KParams& p, const float (&z)[32]) {
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const float z1 = z[2 * i], z2 = z[2 * i + 1];
            fine_dw(p, z1 * p.sqrt_h, fmaf(p.L10, z1, p.L11 * z2) * p.sqrt_h);
            if ((i % MM) == MM - 1) coarse_now(p);
        }
    }
    template <int MM>
    __device__ __forceinline__ void tile_smem_mm(const KParams& p, const float4* row4, int lane) {
#pragma unroll 1
        for (int c2 = 0; c2 < 4; c2++) {
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const float4 v = row4[(2 * c2 + cc) ^ (lane & 7)];
                fine_dw(p, v.x * p.sqrt_h, fmaf(p.L10, v.x, p.L11 * v.y) * p.sqrt_h);
                fine_dw(p, v.z * p.sqrt_h, fmaf(p.L10, v.z, p.L11 * v.w) * p.sqrt_h);
                if (MM == 2 || cc == 1) coarse_now(p);   // after fine steps 2 (M = 2) or 4 (M = 4)
            }
        }
    }
    // raw normals, tile of 32 dimensions starting at a tile boundary
    __device__ __forceinline__ void tile(const KParams& p, const float (&z)[32], int nv) {
        if (nv == 32) {
            if constexpr (HES && COUPLED) {
                if (m == 0 && p.M == 2) {
                    tile_hes_mm<2>(p, z);
                } else if (m == 0 && p.M == 4) {
                    tile_hes_mm<4>(p, z);
                } else {
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        const float z1 = z[2 * i], z2 = z[2 * i + 1];
                        step_dw(p, z1 * p.sqrt_h, fmaf(p.L10, z1, p.L11 * z2) * p.sqrt_h);
                    }
                }
            } else if constexpr (HES) {
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const float z1 = z[2 * i], z2 = z[2 * i + 1];
                    step_dw(p, z1 * p.sqrt_h, fmaf(p.L10, z1, p.L11 * z2) * p.sqrt_h);
                }
            } else if constexpr (MOD == MOD_GBM && !COUPLED) {
                const float sig_sqh = p.sigma * p.sqrt_h;
#pragma unroll
                for (int i = 0; i < 32; i++) f.step_gbm_z(z[i], sig_sqh, muh_f);
                k += 32;
            } else if constexpr (COUPLED) {
                if (m == 0 && p.M == 2) {
                    tile_mm<2>(p, z);
                } else if (m == 0 && p.M == 4) {
                    tile_mm<4>(p, z);
                } else {
#pragma unroll
                    for (int i = 0; i < 32; i++) step_dw(p, z[i] * p.sqrt_h, 0.f);
                }
            } else {
#pragma unroll
                for (int i = 0; i < 32; i++) step_dw(p, z[i] * p.sqrt_h, 0.f);
            }
        } else {
            if constexpr (HES) {
#pragma unroll
                for (int i = 0; i < 16; i++)
                    if (2 * i < nv) {
                        const float z1 = z[2 * i], z2 = z[2 * i + 1];
                        step_dw(p, z1 * p.sqrt_h, fmaf(p.L10, z1, p.L11 * z2) * p.sqrt_h);
                    }
            } else {
#pragma unroll
                for (int i = 0; i < 32; i++)
                    if (i < nv) step_dw(p, z[i] * p.sqrt_h, 0.f);
            }
        }
        flush();
    }
    // Heston: the same steps fed straight from this lane's row of a transposed tile in shared
    // memory, four normals (two steps) per float4 and the chunk loop rolled; the fully unrolled
    // sixteen steps of tile() (fine and coarse legs) weighed on the instruction cache
    static constexpr bool SMEM_TILE = HES;
    __device__ __forceinline__ void tile_smem(const KParams& p, const float* buf, int lane, int nv) {
        const float4* row4 = reinterpret_cast<const float4*>(buf + lane * 32);
        if constexpr (COUPLED) {
            if (nv == 32 && m == 0 && (p.M == 2 || p.M == 4)) {
                if (p.M == 2) tile_smem_mm<2>(p, row4, lane);
                else tile_smem_mm<4>(p, row4, lane);
                flush();
                return;
            }
        }
#pragma unroll 2
        for (int c = 0; c < 8; c++) {
            if (4 * c < nv) {
                const float4 v = row4[c ^ (lane & 7)];
                step_dw(p, v.x * p.sqrt_h, fmaf(p.L10, v.x, p.L11 * v.y) * p.sqrt_h);
                if (4 * c + 2 < nv) step_dw(p, v.z * p.sqrt_h, fmaf(p.L10, v.z, p.L11 * v.w) * p.sqrt_h);
            }
        }
        flush();
    }
    // fold the running partial sums (called at least every 32 steps)
    __device__ __forceinline__ void flush() {
        f.flush();
        if constexpr (COUPLED) c.flush();
    }
    __device__ __forceinline__ void finish(const KParams& p, float (&y)[NST]) {
        flush();
        const float pf = f.payoff(p, p.n_steps, p.corr_f);
        if constexpr (COUPLED) {
            const float pc = (p.n_coarse > 0) ? c.payoff(p, p.n_coarse, p.corr_c) : 0.f;
            const float dy = pf - pc;
            y[0] = dy; y[1] = dy * dy; y[2] = pf; y[3] = pf * pf;
        } else {
            y[0] = pf; y[1] = pf * pf;
        }
    }
};

// Arithmetic Asian with geometric-Asian control on the same GBM path (kernel_gbm_asian_cv,
// methods_cuda.cu:601-640): stats {Ya, Ya^2, Ycv, Ycv^2, Yg, Yg^2, Ya*Yg}.
struct CvAsianC {
    __device__ __forceinline__ void flush() {}
    __device__ __forceinline__ void bind(int, uint64_t) {}
    static constexpr int NST = 7;
    float S, sa, ca, sl, cl, muh;
    __device__ __forceinline__ void init(const KParams& p) {
        S = p.S0; sa = ca = sl = cl = 0.f; muh = p.mu * p.h;
    }
    __device__ __forceinline__ void step_dw(const KParams& p, float dw, float) {
        S = fmaf(S, fmaf(p.sigma, dw, muh), S);
        kadd(sa, ca, S);
        kadd(sl, cl, logf(S));
    }
    __device__ __forceinline__ void tile(const KParams& p, const float (&z)[32], int nv) {
#pragma unroll
        for (int i = 0; i < 32; i++)
            if (i < nv) step_dw(p, z[i] * p.sqrt_h, 0.f);
    }
    __device__ __forceinline__ void finish(const KParams& p, float (&y)[NST]) {
        const float n = (float)p.n_steps;
        const float ya = fmaxf((sa - ca) / n - p.K, 0.f);
        const float yg = fmaxf(expf((sl - cl) / n) - p.K, 0.f);
        const float ycv = ya - p.beta_cv * (yg - p.E_ctrl);
        y[0] = ya; y[1] = ya * ya; y[2] = ycv; y[3] = ycv * ycv;
        y[4] = yg; y[5] = yg * yg; y[6] = ya * yg;
    }
};

// Dupire European with a GBM European control on the same increments
// (kernel_dupire_gbm_cv, methods_cuda.cu:642-677).
struct CvDupireC {
    __device__ __forceinline__ void flush() {}
    __device__ __forceinline__ void bind(int, uint64_t) {}
    static constexpr int NST = 7;
    float Sd, Sg, muh;
    int k;
    __device__ __forceinline__ void init(const KParams& p) {
        Sd = Sg = p.S0; muh = p.mu * p.h; k = 0;
    }
    __device__ __forceinline__ void step_dw(const KParams& p, float dw, float) {
        const float t = (float)k * p.h;
        const float sl = dupire_vol(p, Sd * p.inv_S0, t);
        Sd = fmaf(Sd, fmaf(sl, dw, muh), Sd);
        Sg = fmaf(Sg, fmaf(p.ctrl_sigma, dw, muh), Sg);
        k++;
    }
    __device__ __forceinline__ void tile(const KParams& p, const float (&z)[32], int nv) {
#pragma unroll
        for (int i = 0; i < 32; i++)
            if (i < nv) step_dw(p, z[i] * p.sqrt_h, 0.f);
    }
    __device__ __forceinline__ void finish(const KParams& p, float (&y)[NST]) {
        const float yd = fmaxf(Sd - p.K, 0.f) * p.disc;
        const float yg = fmaxf(Sg - p.K, 0.f) * p.disc;
        const float ycv = yd - p.beta_cv * (yg - p.E_ctrl);
        y[0] = yd; y[1] = yd * yd; y[2] = ycv; y[3] = ycv * ycv;
        y[4] = yg; y[5] = yg * yg; y[6] = yd * yg;
    }
};

// GBM European under the drift-shifted measure Z' = Z + z* with likelihood ratio
// exp(-z* sum Z - N z*^2 / 2) (kernel_is_gbm, methods_cuda.cu:685-707).
struct IsC {
    __device__ __forceinline__ void flush() {}
    __device__ __forceinline__ void bind(int, uint64_t) {}
    static constexpr int NST = 2;
    float S, zs, zc, muh;
    __device__ __forceinline__ void init(const KParams& p) {
        S = p.S0; zs = zc = 0.f; muh = p.mu * p.h;
    }
    __device__ __forceinline__ void tile(const KParams& p, const float (&z)[32], int nv) {
#pragma unroll
        for (int i = 0; i < 32; i++)
            if (i < nv) {
                kadd(zs, zc, z[i]);
                S = fmaf(S, fmaf(p.sigma, (z[i] + p.z_star) * p.sqrt_h, muh), S);
            }
    }
    __device__ __forceinline__ void step_dw(const KParams&, float, float) {}
    __device__ __forceinline__ void finish(const KParams& p, float (&y)[NST]) {
        const float lr = expf(-p.z_star * (zs - zc) - 0.5f * p.z_star * p.z_star * (float)p.n_steps);
        const float v = fmaxf(S - p.K, 0.f) * p.disc * lr;
        y[0] = v; y[1] = v * v;
    }
};

// Multi-asset basket (kernel_multi_dupire, methods_cuda.cu:525-551, with the Cholesky product
// of correlate_multi_dupire :1122-1148 done in registers): dims of step k are k*n + a.
// MOD_MULTI: parametric Dupire per asset; sigma_loc's S0 scale is read per asset from the second
// block of p.bsk (1 / S0 of asset 0 for every asset, the reference's c_p.S0 (:542, :289), or the
// asset's own under MCQ_FLAG_BASKET_OWN_S0); MOD_BASKET: GBM per asset with its own sigma,
// weighted basket.
template <int MOD, int NB>
struct BasketC {
    static constexpr int NST = 2;
    __device__ __forceinline__ void flush() {}
    __device__ __forceinline__ void bind(int, uint64_t) {}
    float S[NB], dw[NB];
    float muh;
    int f, k;
    __device__ __forceinline__ void init(const KParams& p) {
        const int n = p.n_assets;
#pragma unroll
        for (int a = 0; a < NB; a++) { S[a] = (a < n) ? __ldg(p.bsk + a) : 0.f; dw[a] = 0.f; }
        muh = p.mu * p.h;
        f = 0; k = 0;
    }
    __device__ __forceinline__ void feed(const KParams& p, float z) {
        const int n = p.n_assets;
        const float x = z * p.sqrt_h;
        if (p.uncorrelated) {
#pragma unroll
            for (int a = 0; a < NB; a++) if (a == f) dw[a] = x;
        } else {
            const float* Lrow = p.bsk + 3 * n + f;   // L[a][f] at Lrow[a * n]
#pragma unroll
            for (int a = 0; a < NB; a++)
                if (a >= f && a < n) dw[a] = fmaf(__ldg(Lrow + a * n), x, dw[a]);
        }
        if (++f == n) {
            const float t = (float)k * p.h;
#pragma unroll
            for (int a = 0; a < NB; a++) {
                if (a < n) {
                    if constexpr (MOD == MOD_MULTI) {
                        const float sl = dupire_vol(p, S[a] * __ldg(p.bsk + n + a), t);
                        S[a] = fmaf(S[a], fmaf(sl, dw[a], muh), S[a]);
                    } else {
                        S[a] = fmaf(S[a], fmaf(__ldg(p.bsk + n + a), dw[a], muh), S[a]);
                    }
                }
                dw[a] = 0.f;
            }
            f = 0; k++;
        }
    }
    __device__ __forceinline__ void tile(const KParams& p, const float (&z)[32], int nv) {
#pragma unroll
        for (int i = 0; i < 32; i++)
            if (i < nv) feed(p, z[i]);
    }
    __device__ __forceinline__ void step_dw(const KParams&, float, float) {}
    __device__ __forceinline__ void finish(const KParams& p, float (&y)[NST]) {
        const int n = p.n_assets;
        float b = 0.f;
        if constexpr (MOD == MOD_MULTI) {
#pragma unroll
            for (int a = 0; a < NB; a++) if (a < n) b += S[a];
            b = b / (float)n;
        } else {
#pragma unroll
            for (int a = 0; a < NB; a++) if (a < n) b = fmaf(__ldg(p.bsk + 2 * n + a), S[a], b);
        }
        const float v = fmaxf(b - p.K, 0.f) * p.disc;
        y[0] = v; y[1] = v * v;
    }
};

// Parity probe: records the normals (raw) or increments (bridge) the pass consumed for one
// path, so tests can compare the fused generation bit for bit with the reference stream.
struct DumpC {
    __device__ __forceinline__ void flush() {}
    static constexpr int NST = 1;
    float* out;
    int idx;
    bool on;
    __device__ __forceinline__ void init(const KParams&) { idx = 0; }
    __device__ __forceinline__ void bind(const KParams& p, int r, uint64_t n) {
        on = n >= p.offset && n < p.offset + p.n_points;
        out = p.dump + ((size_t)r * p.n_points + (size_t)(n - p.offset)) * (size_t)p.D;
    }
    __device__ __forceinline__ void tile(const KParams&, const float (&z)[32], int nv) {
#pragma unroll
        for (int i = 0; i < 32; i++)
            if (i < nv && on) out[idx + i] = z[i];
        idx += nv;
    }
    __device__ __forceinline__ void step_dw(const KParams&, float dw, float) {
        if (on) out[idx] = dw;
        idx++;
    }
    __device__ __forceinline__ void finish(const KParams&, float (&y)[NST]) { y[0] = 0.f; }
};

// Coupled fine / coarse correlated basket for MLMC / MLQMC levels (the reference refuses
// baskets there, methods_cuda.cu:1318-1320, :1695-1697), with the pathwise delta per asset.
// MOD_BASKET: GBM per asset with its own sigma and a weighted basket.  Euler GBM is linear in
// S0_a, so dS_a(T)/dS0_a = S_a(T)/S0_a and delta_a = disc 1{B > K} w_a S_a(T) / S0_a on each of
// the fine and coarse paths.
// MOD_MULTI: the reference's Dupire basket (parametric local vol per asset, equally weighted
// mean, kernel_multi_dupire :525-551) stepped as kernel_mlmc steps a one-asset Dupire path
// (:471-497): fine steps at t = k h, coarse steps at t = k_c h_c on the summed increments.  Under
// MCQ_FLAG_BASKET_OWN_S0 each asset's volatility is scaled by its own S0, the path is then
// homogeneous of degree one in (S0_a, S_a) and the same delta formula is the total derivative
// dP/dS0_a (the scale inside sigma_loc moving with S0_a, as the one-asset Dupire adjoint); with
// the reference's asset-0 scale it is not, and the deltas are left at 0.
// Statistics: {dY, dY^2, Yf, Yf^2, d delta_0 .. d delta_15}.
template <int MOD, int NB>
struct BasketLevelC {
    static constexpr int NST = 4 + kMaxBasket;
    static constexpr bool WARP_ACC = true;
    float Sf[NB], Sc[NB], dw[NB], acc[NB];
    float muh_f, muh_c;
    int f, m, k, kc;
    __device__ __forceinline__ void bind(int, uint64_t) {}
    __device__ __forceinline__ void flush() {}
    __device__ __forceinline__ void init(const KParams& p) {
        const int n = p.n_assets;
#pragma unroll
        for (int a = 0; a < NB; a++) {
            Sf[a] = Sc[a] = (a < n) ? __ldg(p.bsk + a) : 0.f;
            dw[a] = acc[a] = 0.f;
        }
        muh_f = p.mu * p.h;
        muh_c = p.mu * p.hc;
        f = 0; m = 0; k = 0; kc = 0;
    }
    // sigma_loc(S, t) S-scale: the per-asset inverse reference S0 (second block of p.bsk)
    __device__ __forceinline__ float vol(const KParams& p, int n, int a, float S, float t) const {
        if constexpr (MOD == MOD_MULTI)
            return dupire_vol(p, S * __ldg(p.bsk + n + a), t);
        else
            return __ldg(p.bsk + n + a);
    }
    __device__ __forceinline__ void feed(const KParams& p, float z) {
        const int n = p.n_assets;
        const float x = z * p.sqrt_h;
        if (p.uncorrelated) {
#pragma unroll
            for (int a = 0; a < NB; a++) if (a == f) dw[a] = x;
        } else {
            const float* Lcol = p.bsk + 3 * n + f;
#pragma unroll
            for (int a = 0; a < NB; a++)
                if (a >= f && a < n) dw[a] = fmaf(__ldg(Lcol + a * n), x, dw[a]);
        }
        if (++f == n) {
            const bool coarse = (++m == p.M);
            const float t = (float)k * p.h, tc = (float)kc * p.hc;
#pragma unroll
            for (int a = 0; a < NB; a++) {
                if (a < n) {
                    Sf[a] = fmaf(Sf[a], fmaf(vol(p, n, a, Sf[a], t), dw[a], muh_f), Sf[a]);
                    acc[a] += dw[a];
                    if (coarse) {
                        Sc[a] = fmaf(Sc[a], fmaf(vol(p, n, a, Sc[a], tc), acc[a], muh_c), Sc[a]);
                        acc[a] = 0.f;
                    }
                }
                dw[a] = 0.f;
            }
            if (coarse) { m = 0; kc++; }
            f = 0;
            k++;
        }
    }
    __device__ __forceinline__ void tile(const KParams& p, const float (&z)[32], int nv) {
#pragma unroll
        for (int i = 0; i < 32; i++)
            if (i < nv) feed(p, z[i]);
    }
    __device__ __forceinline__ void step_dw(const KParams&, float, float) {}
    __device__ __forceinline__ void finish(const KParams& p, float (&y)[NST]) {
        const int n = p.n_assets;
        float Bf = 0.f, Bc = 0.f;
        if constexpr (MOD == MOD_MULTI) {   // equally weighted mean, as kernel_multi_dupire
#pragma unroll
            for (int a = 0; a < NB; a++)
                if (a < n) { Bf += Sf[a]; Bc += Sc[a]; }
            Bf = Bf / (float)n;
            Bc = Bc / (float)n;
        } else {
#pragma unroll
            for (int a = 0; a < NB; a++)
                if (a < n) {
                    const float w = __ldg(p.bsk + 2 * n + a);
                    Bf = fmaf(w, Sf[a], Bf);
                    Bc = fmaf(w, Sc[a], Bc);
                }
        }
        const bool has_c = p.n_coarse > 0;
        const float yf = fmaxf(Bf - p.K, 0.f) * p.disc;
        const float yc = has_c ? fmaxf(Bc - p.K, 0.f) * p.disc : 0.f;
        const float dy = yf - yc;
        y[0] = dy; y[1] = dy * dy; y[2] = yf; y[3] = yf * yf;
        const bool deltas = (MOD == MOD_BASKET) || (p.flags & MCQ_FLAG_OWN_S0_CODE);
        const float gf = (Bf > p.K) ? p.disc : 0.f, gc = (has_c && Bc > p.K) ? p.disc : 0.f;
#pragma unroll
        for (int a = 0; a < kMaxBasket; a++) {
            float v = 0.f;
            if (a < NB && a < n && deltas) {
                const float wa = __ldg(p.bsk + 2 * n + a) / __ldg(p.bsk + a);
                v = wa * (gf * Sf[a] - gc * Sc[a]);
            }
            y[4 + a] = v;
        }
    }
};

// Wide basket (up to NMAX assets: kMaxWideBasket for the reference's 100-asset example,
// kMaxHugeBasket for its 1000-asset uncorrelated one): the same arithmetic as BasketC with the
// per-asset state in local memory and rolled loops.
template <int MOD, int NMAX = kMaxWideBasket>
struct BasketWideC {
    static constexpr int NST = 2;
    float S[NMAX], dw[NMAX];
    float muh;
    int f, k;
    __device__ __forceinline__ void bind(int, uint64_t) {}
    __device__ __forceinline__ void flush() {}
    __device__ __forceinline__ void init(const KParams& p) {
        const int n = p.n_assets;
#pragma unroll 1
        for (int a = 0; a < n; a++) { S[a] = __ldg(p.bsk + a); dw[a] = 0.f; }
        muh = p.mu * p.h;
        f = 0; k = 0;
    }
    __device__ __forceinline__ void feed(const KParams& p, float z) {
        const int n = p.n_assets;
        const float x = z * p.sqrt_h;
        if (p.uncorrelated) {
            dw[f] = x;
        } else {
            const float* Lcol = p.bsk + 3 * n + f;
#pragma unroll 1
            for (int a = f; a < n; a++) dw[a] = fmaf(__ldg(Lcol + a * n), x, dw[a]);
        }
        if (++f == n) {
            const float t = (float)k * p.h;
#pragma unroll 1
            for (int a = 0; a < n; a++) {
                if constexpr (MOD == MOD_MULTI) {
                    const float sl = dupire_vol(p, S[a] * __ldg(p.bsk + n + a), t);
                    S[a] = fmaf(S[a], fmaf(sl, dw[a], muh), S[a]);
                } else {
                    S[a] = fmaf(S[a], fmaf(__ldg(p.bsk + n + a), dw[a], muh), S[a]);
                }
                dw[a] = 0.f;
            }
            f = 0; k++;
        }
    }
    __device__ __forceinline__ void tile(const KParams& p, const float (&z)[32], int nv) {
#pragma unroll
        for (int i = 0; i < 32; i++)
            if (i < nv) feed(p, z[i]);
    }
    __device__ __forceinline__ void step_dw(const KParams&, float, float) {}
    __device__ __forceinline__ void finish(const KParams& p, float (&y)[NST]) {
        const int n = p.n_assets;
        float b = 0.f;
        if constexpr (MOD == MOD_MULTI) {
#pragma unroll 1
            for (int a = 0; a < n; a++) b += S[a];
            b = b / (float)n;
        } else {
#pragma unroll 1
            for (int a = 0; a < n; a++) b = fmaf(__ldg(p.bsk + 2 * n + a), S[a], b);
        }
        const float v = fmaxf(b - p.K, 0.f) * p.disc;
        y[0] = v; y[1] = v * v;
    }
};

// ------------------------------------------------------------------ Brownian bridge

// Window of 32 increments from the bridge between W_L = W(32q) and W_R = W(32q + 32):
// 31 interior points over five levels, all indices static.  zs[s] is the normal of interior
// slot s (level u = floor(log2(s+1)), position v = s + 1 - 2^u); its Sobol dimension is
// (S << u) + (q << u) + v (bb_precompute's level order, utils.cpp:78-99) and its weights are
// read from the per-dimension table.
template <bool UNI, class C>
__device__ __forceinline__ void bb_window(const KParams& p, C& cons, const float (&zs)[32],
                                          float WL, float WR, int S, int q) {
    float W[33];
    W[0] = WL;
    W[32] = WR;
#pragma unroll
    for (int u = 0; u < 5; u++) {
#pragma unroll
        for (int v = 0; v < (1 << u); v++) {
            const int s = (1 << u) - 1 + v;
            const int half = 16 >> u;
            const int mid = (2 * v + 1) * half, lft = 2 * v * half, rgt = (2 * v + 2) * half;
            float4 w;
            if constexpr (UNI) {   // level weights from the parameter block: no loads
                w = make_float4(p.bbw[u][0], p.bbw[u][1], p.bbw[u][2], 0.f);
            } else {
                w = __ldg(p.bb + (S << u) + (q << u) + v);
            }
            W[mid] = fmaf(w.x, W[lft], fmaf(w.y, W[rgt], w.z * zs[s]));
        }
    }
#pragma unroll
    for (int t = 0; t < 32; t++) cons.step_dw(p, W[t + 1] - W[t], 0.f);
    cons.flush();
}

// ------------------------------------------------------------------ the pass kernel

template <class C, class = void>
struct smem_tile_of { static constexpr bool value = false; };
template <class C>
struct smem_tile_of<C, std::void_t<decltype(C::SMEM_TILE)>> { static constexpr bool value = C::SMEM_TILE; };

// One 32-path group h of a consumer.  `carry` (nullptr: none) holds the Sobol start words of
// every tile the group generates, slot 32 t + lane for its t-th tile; cont says that the slots
// hold group h - 1's words of the same replica (see sobol_tile).
template <int GEN, int NOISE, class C, int GU = 1>
__device__ __forceinline__ void run_group(const KParams& p, C& cons, const uint32_t* dr,
                                          uint32_t stream, uint64_t h, uint64_t n, float* buf,
                                          float* skel, int lane, uint32_t* carry = nullptr,
                                          bool cont = false) {
    const int D = p.D;
    if constexpr (NOISE == NOISE_RAW) {
        for (int d0 = 0; d0 < D; d0 += 32) {
            float z[32];
            uint32_t* slot = carry ? carry + d0 + lane : nullptr;
            if constexpr (GEN == GEN_SOBOL && smem_tile_of<C>::value) {
                sobol_tile<GU>(dr, p.dstride, d0 + lane, d0 + lane < D, h, p.u_cap, buf, lane, slot, cont);
                __syncwarp();
                cons.tile_smem(p, buf, lane, min(32, D - d0));
                __syncwarp();
                continue;
            } else if constexpr (GEN == GEN_SOBOL) {
                sobol_tile<GU>(dr, p.dstride, d0 + lane, d0 + lane < D, h, p.u_cap, buf, lane, slot, cont);
                __syncwarp();
                read_row(buf, lane, z);
                __syncwarp();
            } else {
                philox_tile(p.seed, stream, n, d0 >> 5, z);
            }
            cons.tile(p, z, min(32, D - d0));
        }
    } else if constexpr (NOISE == NOISE_PCA) {
        // N <= 32 (one tile): dW_i = sum_k M[i][k] z_k with z and M rounded to fp16 as the
        // reference's cast + GEMM (methods_cuda.cu:1228-1229); larger N runs in k_pca.
        const int N = D;
        sobol_tile<GU>(dr, p.dstride, lane, lane < N, h, p.u_cap, buf, lane, carry ? carry + lane : nullptr, cont);
        __syncwarp();
        float z[32];
        read_row(buf, lane, z);
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 32; j++) z[j] = __half2float(__float2half_rn(z[j]));
        const __half* Mrow = static_cast<const __half*>(p.pca);
        for (int i = 0; i < N; i++) {
            float acc = 0.f;
#pragma unroll
            for (int j = 0; j < 32; j++)
                if (j < N) acc = fmaf(__half2float(Mrow[i * N + j]), z[j], acc);
            cons.step_dw(p, acc, 0.f);
        }
        cons.flush();
    } else if constexpr (NOISE == NOISE_DW) {
        // increments produced outside the pass (the large-N PCA product), time-ordered in
        // p.dw_in[i * p.dw_stride + row] for the point offset + row; lanes of a group read
        // consecutive rows (coalesced).  Lanes outside the point range step on zeros.
        const bool valid = n >= p.offset && n < p.offset + p.n_points;
        const float* col = p.dw_in + (valid ? (size_t)(n - p.offset) : (size_t)0);
        for (int t0 = 0; t0 < D; t0 += 32) {
            const int nv = min(32, D - t0);
#pragma unroll 4
            for (int i = 0; i < nv; i++)
                cons.step_dw(p, valid ? __ldg(col + (size_t)(t0 + i) * (size_t)p.dw_stride) : 0.f, 0.f);
            cons.flush();
        }
    } else {   // NOISE_BB, one factor: D == n_steps == N (power of two)
        // Bridge table row j (Sobol dimension j = bb_precompute step j, utils.cpp:54-101):
        // p.bb[j] = {wl, wr, sd, bits(m)} and p.bbi[j] = {l, r}: W[m] = wl W[l] + wr W[r] + sd z_j.
        const int N = D;
        if (N <= 32) {
            // one tile: the literal table-driven bridge (bb_apply, utils.cpp:104-124)
            sobol_tile<GU>(dr, p.dstride, lane, lane < N, h, p.u_cap, buf, lane, carry ? carry + lane : nullptr, cont);
            __syncwarp();
            float z[32];
            read_row(buf, lane, z);
            __syncwarp();
            float W[33];
#pragma unroll
            for (int i = 0; i < 33; i++) W[i] = 0.f;
#pragma unroll
            for (int j = 0; j < 32; j++) {
                if (j < N) {
                    const float4 w = __ldg(p.bb + j);
                    const int2 lr = __ldg(p.bbi + j);
                    W[__float_as_int(w.w)] = fmaf(w.x, W[lr.x], fmaf(w.y, W[lr.y], w.z * z[j]));
                }
            }
#pragma unroll
            for (int t = 0; t < 32; t++)
                if (t < N) cons.step_dw(p, W[t + 1] - W[t], 0.f);
            cons.flush();
        } else {
            // Skeleton W(32q), q = 0..S, from dimensions 0..S-1 (all multiples of 32), kept
            // per lane in shared memory at skel[q * 32 + lane]; then S windows of 32 steps.
            const int S = N >> 5;
            skel[lane] = 0.f;
            // carry slots: the skeleton tiles first, then one per window
            const int ns = (S + 31) & ~31;
            for (int t0 = 0; t0 < S; t0 += 32) {
                sobol_tile<GU>(dr, p.dstride, t0 + lane, t0 + lane < S, h, p.u_cap, buf, lane,
                           carry ? carry + t0 + lane : nullptr, cont);
                __syncwarp();
                float z[32];
                read_row(buf, lane, z);
                __syncwarp();
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    const int dim = t0 + j;
                    if (dim < S) {
                        const float4 w = __ldg(p.bb + dim);
                        const int2 lr = __ldg(p.bbi + dim);
                        const int mi = __float_as_int(w.w) >> 5, li = lr.x >> 5, ri = lr.y >> 5;
                        skel[mi * 32 + lane] = fmaf(w.x, skel[li * 32 + lane],
                                                    fmaf(w.y, skel[ri * 32 + lane], w.z * z[j]));
                    }
                }
            }
            for (int q = 0; q < S; q++) {
                int dim = 0;
                const bool act = lane < 31;
                if (act) {
                    const int u = 31 - __clz(lane + 1);
                    dim = (S << u) + (q << u) + (lane + 1 - (1 << u));
                }
                sobol_tile<GU>(dr, p.dstride, dim, act, h, p.u_cap, buf, lane,
                           carry ? carry + ns + 32 * q + lane : nullptr, cont);
                __syncwarp();
                float z[32];
                read_row(buf, lane, z);
                __syncwarp();
                bb_window<NOISE == NOISE_BB_UNI>(p, cons, z, skel[q * 32 + lane], skel[(q + 1) * 32 + lane], S, q);
            }
        }
    }
}

// ------------------------------------------------------------------ assisted passes

// A pass with few 32-path groups and long paths leaves most of the GPU idle: each warp walks its
// paths' whole step sequence alone, and the generation of its normals stalls the sequential
// path arithmetic it cannot overlap with.  Assisted passes give every path-owning warp three
// helper warps that generate its normal tiles ahead into a four-slot shared-memory ring; the
// owner reads each tile (its own row) and runs the consumer.  The normals, the consumer and the
// work items are those of the plain loop, so the sums are the same bits.  Every wait is bounded;
// a warp that gives up records MCQ_ERR_TIMEOUT in p.err and stops.
constexpr uint32_t kAssistWaitLimit = 1u << 26;

__device__ __forceinline__ uint32_t asst_addr(const void* ptr) { return (uint32_t)__cvta_generic_to_shared(ptr); }
__device__ __forceinline__ void asst_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(asst_addr(bar)) : "memory");
}
__device__ __forceinline__ bool asst_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kAssistWaitLimit) {
    const uint32_t a = asst_addr(bar);
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred q;\n mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n"
            " selp.u32 %0, 1, 0, q;\n}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <int GEN, class C>
__device__ __forceinline__ void assisted_pass(const KParams& p, unsigned char* smem) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int team = wib / kAssistTeam, role = wib - team * kAssistTeam;   // role 0 owns the paths
    float* ring = reinterpret_cast<float*>(smem + team * kAssistTeamBytes);
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + kAssistSlots * 1024);
    uint64_t* empty = full + kAssistSlots;
    if (lane == 0 && role == 0) {
        for (int s = 0; s < kAssistSlots; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(asst_addr(&full[s])), "r"(32));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(asst_addr(&empty[s])), "r"(32));
        }
    }
    __syncthreads();
    const int D = p.D, T = (D + 31) >> 5;   // tiles per path
    const uint64_t gend_all = p.g0 + p.G;
    const int total_teams = gridDim.x * kAssistTeams;
    uint32_t u = 0;   // the team's tile sequence number: tile t of group h in item order
    bool stop = false;
    for (int item = blockIdx.x * kAssistTeams + team; item < p.n_items && !stop; item += total_teams) {
        const int r = item / p.items_per_rep;
        const int j = item - r * p.items_per_rep;
        const uint64_t gb = p.g0 + (uint64_t)j * (uint64_t)p.gpi;
        const uint64_t ge = min(gb + (uint64_t)p.gpi, gend_all);
        if (role == 0) {
            Acc<C::NST> acc;
            acc.zero();
            for (uint64_t h = gb; h < ge && !stop; h++) {
                const uint64_t n = h * 32 + (uint64_t)lane;
                C cons;
                cons.init(p);
                cons.bind(r, n);
                for (int t = 0; t < T; t++, u++) {
                    const int s = (int)(u % kAssistSlots);
                    const bool ok = asst_wait(&full[s], (u / kAssistSlots) & 1u);
                    if (!__all_sync(0xffffffffu, ok)) { stop = true; break; }
                    if constexpr (smem_tile_of<C>::value) {
                        cons.tile_smem(p, ring + s * 1024, lane, min(32, D - 32 * t));
                        asst_arrive(&empty[s]);
                    } else {
                        float z[32];
                        read_row(ring + s * 1024, lane, z);
                        asst_arrive(&empty[s]);
                        cons.tile(p, z, min(32, D - 32 * t));
                    }
                }
                if (stop) break;
                float y[C::NST];
                cons.finish(p, y);
                if (n >= p.offset && n < p.offset + p.n_points) acc.add(y);
            }
            if (!stop) acc.flush(p.partials + (size_t)item * C::NST, lane);
        } else {
            const uint32_t* dr = (GEN == GEN_SOBOL) ? p.dirs + (size_t)r * 33 * (size_t)p.dstride : nullptr;
            const uint32_t stream = p.stream_base + (uint32_t)r;
            for (uint64_t h = gb; h < ge && !stop; h++) {
                for (int t = 0; t < T; t++, u++) {
                    if ((int)(u % kAssistHelpers) != role - 1) continue;
                    const int s = (int)(u % kAssistSlots);
                    const uint32_t use = u / kAssistSlots;
                    if (use > 0) {   // the owner has read this slot's previous tile
                        const bool ok = asst_wait(&empty[s], (use - 1) & 1u);
                        if (!__all_sync(0xffffffffu, ok)) { stop = true; break; }
                    }
                    float* b = ring + s * 1024;
                    if constexpr (GEN == GEN_SOBOL) {
                        sobol_tile(dr, p.dstride, 32 * t + lane, 32 * t + lane < D, h, p.u_cap, b, lane);
                    } else {
                        float z[32];
                        philox_tile(p.seed, stream, h * 32 + (uint64_t)lane, t, z);
                        float4* row = reinterpret_cast<float4*>(b + lane * 32);
#pragma unroll
                        for (int c = 0; c < 8; c++)
                            row[c ^ (lane & 7)] = make_float4(z[4 * c], z[4 * c + 1], z[4 * c + 2], z[4 * c + 3]);
                    }
                    asst_arrive(&full[s]);
                }
            }
        }
    }
    if (stop && lane == 0) atomicExch(p.err, MCQ_ERR_TIMEOUT_CODE);
}

__host__ __device__ constexpr bool noise_is_bb(int noise) { return noise == NOISE_BB || noise == NOISE_BB_UNI; }

// MINB: resident CTAs per SM the register budget is set for (0: 2 for the bridge, whose
// window keeps 33 W values live, kMinBlocks otherwise).  Variants differ only in register
// allocation and scheduling, never in arithmetic, so they produce identical sums.
template <class C>
struct warp_acc_of { static constexpr bool value = false; };
template <int MOD, int NB>
struct warp_acc_of<BasketLevelC<MOD, NB>> { static constexpr bool value = true; };

template <int GEN, int NOISE, class C, int MINB = 0, int GU = 1>
__global__ void __launch_bounds__(kThreads, MINB ? MINB : (noise_is_bb(NOISE) ? 2 : kMinBlocks))
    k_pass(const __grid_constant__ KParams p) {
    extern __shared__ float4 smem4[];
    if constexpr (NOISE == NOISE_ASSIST) {
        assisted_pass<GEN, C>(p, reinterpret_cast<unsigned char*>(smem4));
        return;
    }
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    constexpr bool WACC = warp_acc_of<C>::value;
    const int skel_floats = (noise_is_bb(NOISE) && p.D > 32) ? ((p.D >> 5) + 1) * 32 : 0;
    const int acc_floats = WACC ? ((2 * C::NST + 3) & ~3) : 0;
    float* buf = reinterpret_cast<float*>(smem4) + wib * (1024 + skel_floats + acc_floats + p.carry);
    float* skel = buf + 1024;
    double* wrec = reinterpret_cast<double*>(buf + 1024 + skel_floats);
    uint32_t* carry = p.carry ? reinterpret_cast<uint32_t*>(buf + 1024 + skel_floats + acc_floats) : nullptr;
    const int total_warps = gridDim.x * kWarpsPerBlock;
    const uint64_t gend_all = p.g0 + p.G;
    for (int item = blockIdx.x * kWarpsPerBlock + wib; item < p.n_items; item += total_warps) {
        const int r = item / p.items_per_rep;
        const int j = item - r * p.items_per_rep;
        const uint64_t gb = p.g0 + (uint64_t)j * (uint64_t)p.gpi;
        const uint64_t ge = min(gb + (uint64_t)p.gpi, gend_all);
        const uint32_t* dr = (GEN == GEN_SOBOL) ? p.dirs + (size_t)r * 33 * (size_t)p.dstride : nullptr;
        const uint32_t stream = p.stream_base + (uint32_t)r;
        Acc<WACC ? 1 : C::NST> acc;
        AccWarp<C::NST> wacc;
        if constexpr (WACC) wacc.bind(wrec, lane);
        else acc.zero();
        if constexpr (NOISE == NOISE_PACKED) {
            // Paths of D <= 16 normals: one Sobol tile holds Q = 32 / D groups (lane j makes
            // dimension j mod D of group h + j / D), and each lane then runs its Q paths from the
            // transposed tile.  The normals and the order of the paths are those of the
            // one-group-per-tile loop below; only the idle lanes of its tiles are put to work.
            const int D = p.D, Q = 32 / D;
            const int qj = lane / D, dj = lane - qj * D;
            for (uint64_t h = gb; h < ge; h += (uint64_t)Q) {
                const uint64_t hl = h + (uint64_t)qj;
                sobol_tile(dr, p.dstride, dj, qj < Q && hl < ge, hl, p.u_cap, buf, lane);
                __syncwarp();
                const int nq = (int)min((uint64_t)Q, ge - h);
                for (int q = 0; q < nq; q++) {
                    const uint64_t n = (h + (uint64_t)q) * 32 + (uint64_t)lane;
                    C cons;
                    cons.init(p);
                    cons.bind(r, n);
                    float z[32];
#pragma unroll
                    for (int c = 0; c < 32; c++) z[c] = (c < 16 && c < D) ? buf[swz(lane, q * D + c)] : 0.f;
                    cons.tile(p, z, D);
                    float y[C::NST];
                    cons.finish(p, y);
                    if (n >= p.offset && n < p.offset + p.n_points) acc.add(y);
                }
                __syncwarp();
            }
        } else {
            for (uint64_t h = gb; h < ge; h++) {
                const uint64_t n = h * 32 + (uint64_t)lane;
                C cons;
                cons.init(p);
                if constexpr (std::is_same<C, DumpC>::value) cons.bind(p, r, n);
                else cons.bind(r, n);
                run_group<GEN, NOISE, C, GU>(p, cons, dr, stream, h, n, buf, skel, lane, carry, h != gb);
                float y[C::NST];
                cons.finish(p, y);
                const bool valid = n >= p.offset && n < p.offset + p.n_points;
                if constexpr (WACC) wacc.add(y, valid, lane);
                else if (valid) acc.add(y);
            }
        }
        if constexpr (WACC) wacc.flush(p.partials + (size_t)item * C::NST, lane);
        else acc.flush(p.partials + (size_t)item * C::NST, lane);
    }
}

}  // namespace mcq
