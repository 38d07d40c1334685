/*
 * oracle.c — CPU oracle for the pricing hot path.  TEST INFRASTRUCTURE ONLY.
 *
 * Restates, in plain C (FP64 path arithmetic), the algorithm of the reference
 * QuantGuy3/financial-derivatives-montecarlo so that the CUDA engine can be checked against
 * it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference leg use
 * this file, always as the checker or the timed CPU baseline, never as the product path.
 * See oracle.h for how each part is pinned.
 */
#include "oracle.h"

#include <curand.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ Sobol-HH */

/* splitmix32 — methods_cuda.cu:753-759 (the reference's function is __host__ __device__). */
uint32_t orc_splitmix32(uint32_t x) {
    x += 0x9E3779B9u;
    x = (x ^ (x >> 16)) * 0x21F0AAADu;
    x = (x ^ (x >> 15)) * 0x735A2D97u;
    x = x ^ (x >> 15);
    return x;
}

/* Lower-triangular F2 matrix product, row k MSB-first — methods_cuda.cu:781-795 without the
 * final digital shift.  Row k has a 1 on the diagonal (bit 31-k) and pseudo-random bits
 * strictly above it (bits 31..32-k), seeded by splitmix32(base ^ k). */
uint32_t orc_hh_linear(uint32_t raw, uint32_t base) {
    uint32_t out = 0;
    for (int k = 0; k < 32; k++) {
        uint32_t seed = orc_splitmix32(base ^ (uint32_t)k);
        uint32_t diag = 1u << (31 - k);
        uint32_t mask = (k == 0) ? 0u : (0xFFFFFFFFu << (32 - k));
        uint32_t row = diag | (seed & mask);
        uint32_t bit = (uint32_t)__builtin_popcount(row & raw) & 1u;
        out |= bit << (31 - k);
    }
    return out;
}

/* hh_scramble — methods_cuda.cu:781-795: matrix product then digital shift. */
uint32_t orc_hh_scramble(uint32_t raw, uint32_t base) {
    return orc_hh_linear(raw, base) ^ orc_splitmix32(base ^ 0xA5A5A5A5u);
}

static const uint32_t* g_dirs = NULL;
static int g_ndirs = 0;

/* JoeKuo6 direction vectors, fetched at run time from cuRAND exactly as
 * ensure_sobol_dirvectors_uploaded does (methods_cuda.cu:764-775). */
int orc_dirvectors(const uint32_t** table) {
    if (!g_dirs) {
        curandDirectionVectors32_t* dv = NULL;
        if (curandGetDirectionVectors32(&dv, CURAND_DIRECTION_VECTORS_32_JOEKUO6) !=
            CURAND_STATUS_SUCCESS)
            return 0;
        g_dirs = (const uint32_t*)dv;
        g_ndirs = 20000; /* D_MAX_SOBOL, models.hpp:9 */
    }
    if (table) *table = g_dirs;
    return g_ndirs;
}

/* curand_init(dv, n) + curand(): the state after skipahead(n) is the XOR of the direction
 * words over the set bits of gray(n) = n ^ (n >> 1) (curand_kernel.h skipahead for
 * curandStateSobol32_t); the first curand() returns it. */
uint32_t orc_sobol_raw(const uint32_t* v, uint32_t n) {
    uint32_t g = n ^ (n >> 1), x = 0;
    for (int k = 0; k < 32; k++)
        if (g & (1u << k)) x ^= v[k];
    return x;
}

void orc_sobol_hh_u32_literal(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n,
                              uint32_t* out) {
    const uint32_t* dirs;
    orc_dirvectors(&dirs);
    for (int d = 0; d < nd; d++) {
        int dim = dim0 + d;
        uint32_t base = orc_splitmix32(salt) ^ (uint32_t)dim; /* methods_cuda.cu:819 */
        for (int64_t i = 0; i < n; i++) {
            uint32_t raw = orc_sobol_raw(dirs + (size_t)dim * 32, offset + (uint32_t)i);
            out[(size_t)d * n + i] = orc_hh_scramble(raw, base);
        }
    }
}

/* Pre-scrambled direction words: Lv[k] = hh_linear(v[k]); scrambled(n) = shift ^ XOR over
 * gray(n) of Lv[k].  Bit-identical to the literal form because hh_linear is F2-linear. */
static void prescramble(uint32_t salt, int dim, uint32_t Lv[32], uint32_t* shift) {
    const uint32_t* dirs;
    orc_dirvectors(&dirs);
    uint32_t base = orc_splitmix32(salt) ^ (uint32_t)dim;
    for (int k = 0; k < 32; k++) Lv[k] = orc_hh_linear(dirs[(size_t)dim * 32 + k], base);
    *shift = orc_splitmix32(base ^ 0xA5A5A5A5u);
}

static inline uint32_t scr_direct(const uint32_t Lv[32], uint32_t shift, uint32_t n) {
    uint32_t g = n ^ (n >> 1), x = shift;
    while (g) {
        int k = __builtin_ctz(g);
        x ^= Lv[k];
        g &= g - 1;
    }
    return x;
}

void orc_sobol_hh_u32(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n,
                      uint32_t* out) {
    for (int d = 0; d < nd; d++) {
        uint32_t Lv[32], sh;
        prescramble(salt, dim0 + d, Lv, &sh);
        if (n <= 0) continue;
        uint32_t x = scr_direct(Lv, sh, offset);
        out[(size_t)d * n] = x;
        for (int64_t i = 1; i < n; i++) {
            uint32_t idx = offset + (uint32_t)i;      /* moving idx-1 -> idx flips bit ctz(idx) */
            x ^= Lv[__builtin_ctz(idx)];
            out[(size_t)d * n + i] = x;
        }
    }
}

/* u = ((float)s + 1) * 2^-32 in single precision — methods_cuda.cu:823.  s >= 0xFFFFFF80
 * rounds to u == 1.0f; unless MCQ_FLAG_COMPAT_U_INF is set that one value is moved to the
 * largest float below 1 so that the normal stays finite. */
float orc_u_of(uint32_t s, int flags) {
    volatile float f = (float)s;
    volatile float u = (f + 1.0f) * (1.0f / 4294967296.0f);
    float r = u;
    if (!(flags & MCQ_FLAG_COMPAT_U_INF) && r >= 1.0f) r = 0x1.fffffep-1f;
    return r;
}

/* Wichura (1988), Algorithm AS 241 PPND16: inverse of the standard normal CDF, ~1e-16. */
double orc_ppnd16(double p) {
    double q = p - 0.5, r, val;
    if (fabs(q) <= 0.425) {
        r = 0.180625 - q * q;
        val = q * (((((((r * 2509.0809287301226727 + 33430.575583588128105) * r +
                        67265.770927008700853) * r + 45921.953931549871457) * r +
                      13731.693765509461125) * r + 1971.5909503065514427) * r +
                    133.14166789178437745) * r + 3.387132872796366608) /
              (((((((r * 5226.495278852545925 + 28729.085735721942674) * r +
                    39307.89580009271061) * r + 21213.794301586595867) * r +
                  5394.1960214247511077) * r + 687.1870074920579083) * r +
                42.313330701600911252) * r + 1.0);
        return val;
    }
    r = (q < 0) ? p : 1.0 - p;
    if (r <= 0) return (q < 0) ? -INFINITY : INFINITY;
    r = sqrt(-log(r));
    if (r <= 5.0) {
        r -= 1.6;
        val = (((((((r * 7.7454501427834140764e-4 + 0.0227238449892691845833) * r +
                    0.24178072517745061177) * r + 1.27045825245236838258) * r +
                  3.64784832476320460504) * r + 5.7694972214606914055) * r +
                4.6303378461565452959) * r + 1.42343711074968357734) /
              (((((((r * 1.05075007164441684324e-9 + 5.475938084995344946e-4) * r +
                    0.0151986665636164571966) * r + 0.14810397642748007459) * r +
                  0.68976733498510000455) * r + 1.6763848301838038494) * r +
                2.05319162663775882187) * r + 1.0);
    } else {
        r -= 5.0;
        val = (((((((r * 2.01033439929228813265e-7 + 2.71155556874348757815e-5) * r +
                    0.0012426609473880784386) * r + 0.026532189526576123093) * r +
                  0.29656057182850489123) * r + 1.7848265399172913358) * r +
                5.4637849111641143699) * r + 6.6579046435011037772) /
              (((((((r * 2.04426310338993978564e-15 + 1.4215117583164458887e-7) * r +
                    1.8463183175100546818e-5) * r + 7.868691311456132591e-4) * r +
                  0.0148753612908506148525) * r + 0.13692988092273580531) * r +
                0.59983220655588793769) * r + 1.0);
    }
    return (q < 0) ? -val : val;
}

void orc_sobol_hh_normal(uint32_t salt, int dim0, int nd, uint32_t offset, int64_t n,
                         int flags, double* out) {
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)nd * (size_t)(n > 0 ? n : 1));
    orc_sobol_hh_u32(salt, dim0, nd, offset, n, tmp);
    for (int64_t i = 0; i < (int64_t)nd * n; i++) out[i] = orc_ppnd16((double)orc_u_of(tmp[i], flags));
    free(tmp);
}

/* ------------------------------------------------------------------ Philox */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 10 rounds of the 4x32 S-box with
 * multipliers 0xD2511F53 / 0xCD9E8D57 and Weyl key increments 0x9E3779B9 / 0xBB67AE85. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Engine convention for pseudo-random normals of one path: block b of dimensions
 * 4b..4b+3 uses counter {b, path_lo, path_hi, stream} and key {seed, 0x6D637121};
 * each word pair (x, y) gives a Box–Muller pair with u = ((w >> 8) + 0.5) * 2^-24. */
void orc_philox_normals(uint32_t seed, uint32_t stream, uint64_t path, int n, double* z) {
    uint32_t key[2] = {seed, 0x6D637121u};
    for (int b = 0; 4 * b < n; b++) {
        uint32_t ctr[4] = {(uint32_t)b, (uint32_t)path, (uint32_t)(path >> 32), stream}, o[4];
        orc_philox4x32_10(ctr, key, o);
        for (int j = 0; j < 2; j++) {
            float u1 = ((float)(o[2 * j] >> 8) + 0.5f) * (1.0f / 16777216.0f);
            float u2 = ((float)(o[2 * j + 1] >> 8) + 0.5f) * (1.0f / 16777216.0f);
            double rr = sqrt(-2.0 * log((double)u1));
            double a = 2.0 * M_PI * (double)u2;
            int i0 = 4 * b + 2 * j;
            if (i0 < n) z[i0] = rr * sin(a);
            if (i0 + 1 < n) z[i0 + 1] = rr * cos(a);
        }
    }
}

/* ------------------------------------------------------------------ Brownian bridge */

/* bb_precompute — utils.cpp:54-101: step 0 is W[N] with sd sqrt(T); level-order midpoints. */
int orc_bb_precompute(int N, double T, int* map_idx, int* left_idx, int* right_idx, double* wl,
                      double* wr, double* sd) {
    if (N <= 0 || (N & (N - 1))) return -1;
    for (int i = 0; i < N; i++) { map_idx[i] = left_idx[i] = right_idx[i] = 0; wl[i] = wr[i] = sd[i] = 0; }
    map_idx[0] = N;
    sd[0] = sqrt(T);
    int step = 1, levels = 0;
    for (int t = N; t > 1; t >>= 1) levels++;
    for (int lev = 0; lev < levels; lev++) {
        int np = 1 << lev, stride = N >> lev, half = stride >> 1;
        for (int j = 0; j < np; j++) {
            int L = j * stride, R = (j + 1) * stride, M = L + half;
            double tL = L * T / N, tR = R * T / N, tM = M * T / N;
            map_idx[step] = M; left_idx[step] = L; right_idx[step] = R;
            wl[step] = (tR - tM) / (tR - tL);
            wr[step] = (tM - tL) / (tR - tL);
            sd[step] = sqrt((tM - tL) * (tR - tM) / (tR - tL));
            step++;
        }
    }
    return 0;
}

/* bb_apply — utils.cpp:104-124, one path. */
void orc_bb_apply(int N, const int* map_idx, const int* left_idx, const int* right_idx,
                  const double* wl, const double* wr, const double* sd, const double* z,
                  double* dW) {
    double* W = (double*)calloc((size_t)N + 1, sizeof(double));
    W[map_idx[0]] = sd[0] * z[0];
    for (int s = 1; s < N; s++)
        W[map_idx[s]] = wl[s] * W[left_idx[s]] + wr[s] * W[right_idx[s]] + sd[s] * z[s];
    for (int k = 0; k < N; k++) dW[k] = W[k + 1] - W[k];
    free(W);
}

/* ------------------------------------------------------------------ PCA */

/* pca_compute — utils.cpp:131-167.  C_ij = h min(i+1, j+1) has the closed-form eigenpairs
 * lambda_k = h / (4 sin^2((2k+1) pi / (2(2m+1)))), v_k[i] = 2/sqrt(2m+1) sin((2k+1)(i+1) pi/(2m+1)),
 * k = 0.. in descending eigenvalue order; the sign is fixed by v_k[0] > 0.  M_cum = V sqrt(L),
 * M_pca = row difference of M_cum (utils.cpp:151-157).  Column-major m x m. */
int orc_pca_compute(int m, double T, double* M) {
    if (m <= 0) return -1;
    double h = T / m, den = 2.0 * m + 1.0;
    for (int k = 0; k < m; k++) {
        double s = sin((2.0 * k + 1.0) * M_PI / (2.0 * den));
        double lam = h / (4.0 * s * s);
        double sl = sqrt(lam), c = 2.0 / sqrt(den), prev = 0.0;
        for (int i = 0; i < m; i++) {
            double cum = c * sin((2.0 * k + 1.0) * (i + 1.0) * M_PI / den) * sl;
            M[(size_t)k * m + i] = cum - prev;
            prev = cum;
        }
    }
    return 0;
}

/* Cyclic Jacobi eigen-solver on C (numeric cross-check of the closed form). */
int orc_pca_jacobi(int m, double T, double* M) {
    double h = T / m;
    double* A = (double*)malloc(sizeof(double) * m * m);
    double* V = (double*)calloc((size_t)m * m, sizeof(double));
    for (int i = 0; i < m; i++) {
        V[i * m + i] = 1.0;
        for (int j = 0; j < m; j++) A[i * m + j] = h * (double)((i < j ? i : j) + 1);
    }
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0;
        for (int i = 0; i < m; i++)
            for (int j = i + 1; j < m; j++) off += A[i * m + j] * A[i * m + j];
        if (off < 1e-30) break;
        for (int p = 0; p < m; p++)
            for (int q = p + 1; q < m; q++) {
                double apq = A[p * m + q];
                if (fabs(apq) < 1e-300) continue;
                double th = (A[q * m + q] - A[p * m + p]) / (2 * apq);
                double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1));
                double c = 1 / sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < m; k++) {
                    double akp = A[k * m + p], akq = A[k * m + q];
                    A[k * m + p] = c * akp - s * akq;
                    A[k * m + q] = s * akp + c * akq;
                }
                for (int k = 0; k < m; k++) {
                    double apk = A[p * m + k], aqk = A[q * m + k];
                    A[p * m + k] = c * apk - s * aqk;
                    A[q * m + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < m; k++) {
                    double vkp = V[k * m + p], vkq = V[k * m + q];
                    V[k * m + p] = c * vkp - s * vkq;
                    V[k * m + q] = s * vkp + c * vkq;
                }
            }
    }
    int* ord = (int*)malloc(sizeof(int) * m);
    for (int i = 0; i < m; i++) ord[i] = i;
    for (int i = 0; i < m; i++)
        for (int j = i + 1; j < m; j++)
            if (A[ord[j] * m + ord[j]] > A[ord[i] * m + ord[i]]) { int t = ord[i]; ord[i] = ord[j]; ord[j] = t; }
    for (int k = 0; k < m; k++) {
        int e = ord[k];
        double lam = A[e * m + e];
        double sl = sqrt(lam > 0 ? lam : 0), sg = V[0 * m + e] >= 0 ? 1.0 : -1.0, prev = 0;
        for (int i = 0; i < m; i++) {
            double cum = sg * V[i * m + e] * sl;
            M[(size_t)k * m + i] = cum - prev;
            prev = cum;
        }
    }
    free(ord); free(A); free(V);
    return 0;
}

/* ------------------------------------------------------------------ closed forms */

static double ncdf(double x) { return 0.5 * erfc(-x / sqrt(2.0)); }

/* bs_call — utils.cpp:22-28 */
double orc_bs_call(double S0, double K, double T, double r, double sigma) {
    if (T <= 0.0 || sigma <= 0.0) { double v = S0 - K * exp(-r * T); return v > 0 ? v : 0; }
    double sT = sqrt(T);
    double d1 = (log(S0 / K) + (r + 0.5 * sigma * sigma) * T) / (sigma * sT);
    double d2 = d1 - sigma * sT;
    return S0 * ncdf(d1) - K * exp(-r * T) * ncdf(d2);
}

/* geom_asian_analytic — utils.cpp:34-47 (undiscounted, average of S_1..S_n). */
double orc_geom_asian(double S0, double K, double T, double mu, double sigma, int n) {
    double mG = log(S0) + (mu - 0.5 * sigma * sigma) * T * (n + 1) / (2.0 * n);
    double s2 = sigma * sigma * T * (n + 1) * (2.0 * n + 1) / (6.0 * n * n);
    double sG = sqrt(s2);
    if (sG < 1e-12) { double v = exp(mG) - K; return v > 0 ? v : 0; }
    double d1 = (mG + s2 - log(K)) / sG, d2 = d1 - sG;
    return exp(mG + 0.5 * s2) * ncdf(d1) - K * ncdf(d2);
}

/* Continuously monitored down-and-out call under GBM with B <= K (Merton 1973 /
 * Reiner–Rubinstein 1991): C - (B/S)^(2r/sigma^2 - 1) C(B^2/S). */
double orc_down_out_call(double S0, double K, double B, double T, double r, double sigma) {
    if (S0 <= B) return 0.0;
    double c = orc_bs_call(S0, K, T, r, sigma);
    double a = 2.0 * r / (sigma * sigma) - 1.0;
    return c - pow(B / S0, a) * orc_bs_call(B * B / S0, K, T, r, sigma);
}

/* ------------------------------------------------------------------ path arithmetic */

int orc_noise_dim(const mcq_model* m) {   /* model_noise_dim, models.hpp:78-87 */
    switch (m->kind) {
        case MCQ_MODEL_HESTON: return 2;
        case MCQ_MODEL_MULTI_DUPIRE:
        case MCQ_MODEL_BASKET_GBM: return m->n_assets;
        default: return 1;
    }
}

static double pay_discount(const mcq_payoff* p) {   /* make_params, methods_cuda.cu:994-1025 */
    switch (p->kind) {
        case MCQ_PAYOFF_EUROPEAN: case MCQ_PAYOFF_BARRIER_UP_OUT:
        case MCQ_PAYOFF_BARRIER_DOWN_OUT: case MCQ_PAYOFF_BASKET:
            return exp(-p->r * p->T);
        default: return 1.0;
    }
}

static double run_init(const mcq_payoff* p, double S0) {   /* d_running_init, :298-302 */
    if (p->kind == MCQ_PAYOFF_LOOKBACK || p->kind == MCQ_PAYOFF_BARRIER_DOWN_OUT) return S0;
    return 0.0;
}

static void run_update(const mcq_payoff* p, double* run, double S) {   /* :307-312 */
    switch (p->kind) {
        case MCQ_PAYOFF_ASIAN: *run += S; break;
        case MCQ_PAYOFF_GEOM_ASIAN: *run += log(S); break;
        case MCQ_PAYOFF_LOOKBACK: case MCQ_PAYOFF_BARRIER_DOWN_OUT: *run = fmin(*run, S); break;
        case MCQ_PAYOFF_BARRIER_UP_OUT: *run = fmax(*run, S); break;
        default: break;
    }
}

static int path_dep(const mcq_payoff* p) {
    return p->kind == MCQ_PAYOFF_ASIAN || p->kind == MCQ_PAYOFF_GEOM_ASIAN ||
           p->kind == MCQ_PAYOFF_LOOKBACK || p->kind == MCQ_PAYOFF_BARRIER_UP_OUT ||
           p->kind == MCQ_PAYOFF_BARRIER_DOWN_OUT;
}

/* d_apply_bgk — :326-331, with the reference's single-precision constant 0.5826f. */
static void apply_bgk(const mcq_payoff* p, double* run, double h) {
    if (!(p->kind == MCQ_PAYOFF_LOOKBACK || p->kind == MCQ_PAYOFF_BARRIER_UP_OUT ||
          p->kind == MCQ_PAYOFF_BARRIER_DOWN_OUT))
        return;
    double corr = exp(-(double)0.5826f * p->sigma * sqrt(h));
    if (p->kind == MCQ_PAYOFF_BARRIER_UP_OUT) *run /= corr;
    else *run *= corr;
}

/* d_payoff — :335-352 (+ down-and-out) */
static double payoff_value(const mcq_payoff* p, double S, double run, int n) {
    double disc = pay_discount(p);
    switch (p->kind) {
        case MCQ_PAYOFF_EUROPEAN: case MCQ_PAYOFF_BASKET: return fmax(S - p->K, 0.0) * disc;
        case MCQ_PAYOFF_ASIAN: return fmax(run / n - p->K, 0.0);
        case MCQ_PAYOFF_GEOM_ASIAN: return fmax(exp(run / n) - p->K, 0.0);
        case MCQ_PAYOFF_LOOKBACK: return S - run;
        case MCQ_PAYOFF_BARRIER_UP_OUT: return (run >= p->B) ? 0.0 : fmax(S - p->K, 0.0) * disc;
        case MCQ_PAYOFF_BARRIER_DOWN_OUT: return (run <= p->B) ? 0.0 : fmax(S - p->K, 0.0) * disc;
    }
    return 0.0;
}

static double lv_sigma(const mcq_model* m, double S, double t) {
    int nK = m->lv_nK, nt = m->lv_nt;
    const double *Kg = m->lv_K, *tg = m->lv_t;
    double x = S < Kg[0] ? Kg[0] : (S > Kg[nK - 1] ? Kg[nK - 1] : S);
    double y = t < tg[0] ? tg[0] : (t > tg[nt - 1] ? tg[nt - 1] : t);
    int i = 0, j = 0;
    while (i < nK - 2 && Kg[i + 1] <= x) i++;
    while (j < nt - 2 && tg[j + 1] <= y) j++;
    double a = (x - Kg[i]) / (Kg[i + 1] - Kg[i]);
    double b = (y - tg[j]) / (tg[j + 1] - tg[j]);
    const double* s = m->lv_sigma;
    return (1 - a) * (1 - b) * s[j * nK + i] + a * (1 - b) * s[j * nK + i + 1] +
           (1 - a) * b * s[(j + 1) * nK + i] + a * b * s[(j + 1) * nK + i + 1];
}

/* Normals of one path -> time-ordered increments dW[k * d + f]. */
static void make_increments(const mcq_model* m, int n_steps, const orc_noise* nz,
                            const double* z, double* dW) {
    int d = orc_noise_dim(m), D = n_steps * d;
    double sqh = sqrt(m->T / n_steps);
    int mode = nz ? nz->mode : MCQ_NOISE_RAW;
    if (mode == MCQ_NOISE_BB) {
        orc_bb_apply(n_steps, nz->map_idx, nz->left_idx, nz->right_idx, nz->wl, nz->wr, nz->sd,
                     z, dW);
    } else if (mode == MCQ_NOISE_PCA) {
        for (int i = 0; i < n_steps; i++) {
            double acc = 0;
            for (int k = 0; k < n_steps; k++) {
                double a = nz->M_pca[(size_t)k * n_steps + i], b = z[k];
                if (nz->pca_fp16) { a = (double)(_Float16)(float)a; b = (double)(_Float16)(float)b; }
                acc += a * b;
            }
            dW[i] = acc;
        }
    } else {
        for (int i = 0; i < D; i++) dW[i] = z[i] * sqh;
    }
}

/* kernel_mc / d_step / kernel_multi_dupire (methods_cuda.cu:388-437, 525-551) in FP64. */
double orc_path_payoff(const mcq_model* m, const mcq_payoff* p, int n_steps,
                       const orc_noise* nz, const double* z) {
    return orc_path_payoff_f(m, p, n_steps, nz, z, 0);
}

/* as orc_path_payoff; flags & MCQ_FLAG_HESTON_MILSTEIN adds the Milstein term
   xi^2/4 (dW2^2 - h) to the Heston variance step */
double orc_path_payoff_f(const mcq_model* m, const mcq_payoff* p, int n_steps,
                         const orc_noise* nz, const double* z, int flags) {
    int d = orc_noise_dim(m), D = n_steps * d;
    double h = m->T / n_steps;
    double* dW = (double*)malloc(sizeof(double) * D);
    make_increments(m, n_steps, nz, z, dW);
    double Y = 0.0;
    if (m->kind == MCQ_MODEL_MULTI_DUPIRE || m->kind == MCQ_MODEL_BASKET_GBM) {
        int n = m->n_assets;
        double* Sa = (double*)malloc(sizeof(double) * n);
        double* dwc = (double*)malloc(sizeof(double) * n);
        for (int a = 0; a < n; a++) Sa[a] = m->S0_vec ? m->S0_vec[a] : m->S0;
        double S0ref = m->S0_vec ? m->S0_vec[0] : m->S0;   /* c_p.S0 = S0[0], :1046 */
        int own = (flags & MCQ_FLAG_BASKET_OWN_S0) != 0;   /* each asset's own S0 in sigma_loc */
        for (int k = 0; k < n_steps; k++) {
            for (int a = 0; a < n; a++) {
                double acc = 0;
                if (m->uncorrelated || !m->L) acc = dW[k * n + a];
                else for (int j = 0; j <= a; j++) acc += m->L[a * n + j] * dW[k * n + j];
                dwc[a] = acc;
            }
            for (int a = 0; a < n; a++) {
                double S = Sa[a];
                if (m->kind == MCQ_MODEL_MULTI_DUPIRE) {
                    double s0 = own ? m->S0_vec[a] : S0ref;
                    double sl = m->sigma0 * exp(-m->alpha * (k * h)) * pow(S / s0, m->beta_d - 1.0);
                    Sa[a] = S + m->mu * S * h + sl * S * dwc[a];
                } else {
                    Sa[a] = S + m->mu * S * h + m->sigma_vec[a] * S * dwc[a];
                }
            }
        }
        double B = 0;
        for (int a = 0; a < n; a++) B += (m->weights ? m->weights[a] : 1.0 / n) * Sa[a];
        Y = fmax(B - p->K, 0.0) * pay_discount(p);
        free(Sa); free(dwc);
    } else {
        double S = m->S0, V = m->v0, run = run_init(p, m->S0);
        double em = exp(-m->kappa * h);
        for (int k = 0; k < n_steps; k++) {
            switch (m->kind) {
                case MCQ_MODEL_GBM: S = S + m->mu * S * h + m->sigma * S * dW[k]; break;
                case MCQ_MODEL_DUPIRE: {
                    double sl = m->sigma0 * exp(-m->alpha * (k * h)) * pow(S / m->S0, m->beta_d - 1.0);
                    S = S + m->mu * S * h + sl * S * dW[k];
                } break;
                case MCQ_MODEL_LOCALVOL_GRID: {
                    double sl = lv_sigma(m, S, k * h);
                    S = S + m->mu * S * h + sl * S * dW[k];
                } break;
                case MCQ_MODEL_HESTON: {
                    double z1 = dW[2 * k], z2 = dW[2 * k + 1];
                    double dw1 = z1, dw2 = m->hes_L10 * z1 + m->hes_L11 * z2;
                    double Vp = V > 0 ? V : 0, sq = sqrt(Vp);
                    S = S + m->mu * S * h + sq * S * dw1;
                    V = m->theta + em * (V - m->theta) + m->xi * sq * dw2;
                    if (flags & MCQ_FLAG_HESTON_MILSTEIN) V += 0.25 * m->xi * m->xi * (dw2 * dw2 - h);
                } break;
            }
            if (path_dep(p)) run_update(p, &run, S);
        }
        if (path_dep(p)) apply_bgk(p, &run, h);
        Y = payoff_value(p, S, run, n_steps);
    }
    free(dW);
    return Y;
}

/* kernel_mlmc (methods_cuda.cu:445-518) in FP64.  Level 0 (no coarse path) has M coarse
 * steps never completing a payoff: the caller passes n_fine == n0 and Yc = 0 is returned
 * when n_fine < M or the level is 0 (signalled by M <= 0). */
double orc_level_payoff(const mcq_model* m, const mcq_payoff* p, int n_fine, int M,
                        const orc_noise* nz, const double* z, int flags, double* yc) {
    int coarse = M > 0;
    int Mr = coarse ? M : 1;
    int n_coarse = coarse ? n_fine / Mr : 0;
    double T = m->T, hf = T / n_fine, hc = T / (n_coarse > 0 ? n_coarse : 1);
    int d = orc_noise_dim(m), D = n_fine * d;
    double* dW = (double*)malloc(sizeof(double) * D);
    make_increments(m, n_fine, nz, z, dW);
    double Sf = m->S0, Vf = m->v0, Sc = Sf, Vc = Vf;
    double rf = run_init(p, m->S0), rc = rf, a1 = 0, a2 = 0;
    int ck = 0, pd = path_dep(p);
    int skip_hes = (m->kind == MCQ_MODEL_HESTON) && (flags & MCQ_FLAG_COMPAT_HESTON_MLMC);
    double emf = exp(-m->kappa * hf), emc = exp(-m->kappa * hc);
    for (int k = 0; k < n_fine; k++) {
        if (m->kind == MCQ_MODEL_HESTON) {
            double z1 = dW[2 * k], z2 = dW[2 * k + 1];
            double dw1 = z1, dw2 = m->hes_L10 * z1 + m->hes_L11 * z2;
            a1 += dw1; a2 += dw2;
            double Vp = Vf > 0 ? Vf : 0, sq = sqrt(Vp);
            Sf = Sf + m->mu * Sf * hf + sq * Sf * dw1;
            Vf = m->theta + emf * (Vf - m->theta) + m->xi * sq * dw2;
            if (flags & MCQ_FLAG_HESTON_MILSTEIN) Vf += 0.25 * m->xi * m->xi * (dw2 * dw2 - hf);
        } else {
            double dw = dW[k];
            a1 += dw;
            if (m->kind == MCQ_MODEL_GBM) Sf = Sf + m->mu * Sf * hf + m->sigma * Sf * dw;
            else if (m->kind == MCQ_MODEL_DUPIRE) {
                double sl = m->sigma0 * exp(-m->alpha * (k * hf)) * pow(Sf / m->S0, m->beta_d - 1.0);
                Sf = Sf + m->mu * Sf * hf + sl * Sf * dw;
            } else if (m->kind == MCQ_MODEL_LOCALVOL_GRID) {
                double sl = lv_sigma(m, Sf, k * hf);
                Sf = Sf + m->mu * Sf * hf + sl * Sf * dw;
            }
        }
        if (pd && !skip_hes) run_update(p, &rf, Sf);
        if (coarse && (k + 1) % Mr == 0) {
            if (m->kind == MCQ_MODEL_HESTON) {
                double Vp = Vc > 0 ? Vc : 0, sq = sqrt(Vp);
                Sc = Sc + m->mu * Sc * hc + sq * Sc * a1;
                Vc = m->theta + emc * (Vc - m->theta) + m->xi * sq * a2;
                if (flags & MCQ_FLAG_HESTON_MILSTEIN) Vc += 0.25 * m->xi * m->xi * (a2 * a2 - hc);
            } else if (m->kind == MCQ_MODEL_GBM) {
                Sc = Sc + m->mu * Sc * hc + m->sigma * Sc * a1;
            } else if (m->kind == MCQ_MODEL_DUPIRE) {
                double sl = m->sigma0 * exp(-m->alpha * (ck * hc)) * pow(Sc / m->S0, m->beta_d - 1.0);
                Sc = Sc + m->mu * Sc * hc + sl * Sc * a1;
            } else if (m->kind == MCQ_MODEL_LOCALVOL_GRID) {
                double sl = lv_sigma(m, Sc, ck * hc);
                Sc = Sc + m->mu * Sc * hc + sl * Sc * a1;
            }
            if (pd && !skip_hes) run_update(p, &rc, Sc);
            a1 = a2 = 0;
            ck++;
        }
    }
    if (pd) { apply_bgk(p, &rf, hf); apply_bgk(p, &rc, hc); }
    double pf = payoff_value(p, Sf, rf, n_fine);
    double pc = (n_coarse > 0) ? payoff_value(p, Sc, rc, n_coarse) : 0.0;
    free(dW);
    *yc = pc;
    return pf;
}

/* ------------------------------------------------------------------ drivers */

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

#define ORC_CHUNKS 64   /* fixed work split -> results independent of thread count */

int orc_qmc_sums(const mcq_model* m, const mcq_payoff* p, int n_steps, const orc_noise* nz,
                 uint32_t salt_base, int R, uint32_t offset, int64_t N, int flags,
                 int n_threads, double* sums) {
    int D = n_steps * orc_noise_dim(m);
    if (D > 20000) return -1;
    if ((uint64_t)offset + (uint64_t)N > 0x100000000ull) return -2;
    int nch = (N < ORC_CHUNKS) ? (int)(N > 0 ? N : 1) : ORC_CHUNKS;
    double* part = (double*)calloc((size_t)R * nch * 2, sizeof(double));
    uint32_t* Lv = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)R * D * 33);
    for (int r = 0; r < R; r++)
        for (int dd = 0; dd < D; dd++) {
            uint32_t* w = Lv + ((size_t)r * D + dd) * 33;
            prescramble(salt_base + (uint32_t)r, dd, w, w + 32);
        }
    int nt = n_threads > 0 ? n_threads : orc_max_threads();
    (void)nt;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t task = 0; task < (int64_t)R * nch; task++) {
        int r = (int)(task / nch), c = (int)(task % nch);
        int64_t b = N * c / nch, e = N * (c + 1) / nch;
        if (b >= e) continue;
        uint32_t* x = (uint32_t*)malloc(sizeof(uint32_t) * D);
        double* z = (double*)malloc(sizeof(double) * D);
        const uint32_t* L = Lv + (size_t)r * D * 33;
        for (int dd = 0; dd < D; dd++) x[dd] = scr_direct(L + dd * 33, L[dd * 33 + 32], offset + (uint32_t)b);
        double s1 = 0, s2 = 0;
        for (int64_t i = b; i < e; i++) {
            uint32_t idx = offset + (uint32_t)i;
            if (i > b) {
                int k = __builtin_ctz(idx);
                for (int dd = 0; dd < D; dd++) x[dd] ^= L[dd * 33 + k];
            }
            for (int dd = 0; dd < D; dd++) z[dd] = orc_ppnd16((double)orc_u_of(x[dd], flags));
            double y = orc_path_payoff_f(m, p, n_steps, nz, z, flags);
            s1 += y; s2 += y * y;
        }
        part[task * 2] = s1; part[task * 2 + 1] = s2;
        free(x); free(z);
    }
    for (int r = 0; r < R; r++) {
        double a = 0, b2 = 0;
        for (int c = 0; c < nch; c++) { a += part[((size_t)r * nch + c) * 2]; b2 += part[((size_t)r * nch + c) * 2 + 1]; }
        sums[r * 2] = a; sums[r * 2 + 1] = b2;
    }
    free(part); free(Lv);
    return 0;
}

int orc_level_sums(const mcq_model* m, const mcq_payoff* p, int n_fine, int M,
                   const orc_noise* nz, int use_sobol, uint32_t seed, uint32_t salt_base,
                   int R, uint32_t offset, int64_t N, int flags, int n_threads, double* sums) {
    int D = n_fine * orc_noise_dim(m);
    if (use_sobol && D > 20000) return -1;
    int nch = (N < ORC_CHUNKS) ? (int)(N > 0 ? N : 1) : ORC_CHUNKS;
    double* part = (double*)calloc((size_t)R * nch * 4, sizeof(double));
    uint32_t* Lv = NULL;
    if (use_sobol) {
        Lv = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)R * D * 33);
        for (int r = 0; r < R; r++)
            for (int dd = 0; dd < D; dd++) {
                uint32_t* w = Lv + ((size_t)r * D + dd) * 33;
                prescramble(salt_base + (uint32_t)r, dd, w, w + 32);
            }
    }
    int nt = n_threads > 0 ? n_threads : orc_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t task = 0; task < (int64_t)R * nch; task++) {
        int r = (int)(task / nch), c = (int)(task % nch);
        int64_t b = N * c / nch, e = N * (c + 1) / nch;
        if (b >= e) continue;
        uint32_t* x = (uint32_t*)malloc(sizeof(uint32_t) * D);
        double* z = (double*)malloc(sizeof(double) * D);
        const uint32_t* L = use_sobol ? Lv + (size_t)r * D * 33 : NULL;
        if (use_sobol)
            for (int dd = 0; dd < D; dd++) x[dd] = scr_direct(L + dd * 33, L[dd * 33 + 32], offset + (uint32_t)b);
        double s[4] = {0, 0, 0, 0};
        for (int64_t i = b; i < e; i++) {
            uint32_t idx = offset + (uint32_t)i;
            if (use_sobol) {
                if (i > b) { int k = __builtin_ctz(idx); for (int dd = 0; dd < D; dd++) x[dd] ^= L[dd * 33 + k]; }
                for (int dd = 0; dd < D; dd++) z[dd] = orc_ppnd16((double)orc_u_of(x[dd], flags));
            } else {
                orc_philox_normals(seed, salt_base + (uint32_t)r, (uint64_t)offset + (uint64_t)i, D, z);
            }
            double yc, yf = orc_level_payoff(m, p, n_fine, M, nz, z, flags, &yc);
            double dy = yf - yc;
            s[0] += dy; s[1] += dy * dy; s[2] += yf; s[3] += yf * yf;
        }
        for (int q = 0; q < 4; q++) part[task * 4 + q] = s[q];
        free(x); free(z);
    }
    for (int r = 0; r < R; r++)
        for (int q = 0; q < 4; q++) {
            double a = 0;
            for (int c = 0; c < nch; c++) a += part[((size_t)r * nch + c) * 4 + q];
            sums[r * 4 + q] = a;
        }
    free(part); free(Lv);
    return 0;
}

/* Coupled fine/coarse pair of a correlated GBM basket call (per-asset sigma; the correlated
 * increments L z sqrt(h) of correlate_multi_dupire, methods_cuda.cu:1097-1148; fine and coarse
 * paths driven by the same increments as kernel_mlmc, :445-518) in FP64, with the pathwise
 * sensitivities to each S0_a.  Euler is linear in S0_a, so dS_a(T)/dS0_a = S_a(T)/S0_a and
 * d payoff/dS0_a = disc 1{B > K} w_a S_a(T)/S0_a.  z: normals in order step * n + asset.
 * M <= 0: level 0 (no coarse path).  Returns Yf; *yc = Yc; dd[a] = d(Yf - Yc)/dS0_a. */
double orc_basket_level(const mcq_model* m, const mcq_payoff* p, int n_fine, int M, const double* z,
                        double* yc, double* dd) {
    return orc_basket_level_f(m, p, n_fine, M, z, yc, dd, 0);
}

/* The coupled basket pair for the correlated GBM basket (weighted, per-asset sigma) and the
 * reference's Dupire basket (equally weighted mean, sigma_loc with asset 0's S0, or each asset's
 * own under MCQ_FLAG_BASKET_OWN_S0), stepped as kernel_mlmc steps one Dupire path
 * (methods_cuda.cu:471-497: fine steps at t = k h, coarse steps at t = k_c h_c on the summed
 * increments).  dd[a] = w_a / S0_a (gf Sf_a - gc Sc_a): the pathwise dP/dS0_a of the GBM basket,
 * and of the Dupire basket under MCQ_FLAG_BASKET_OWN_S0 (the path is then homogeneous in
 * (S0_a, S_a)); 0 for the Dupire basket with the reference's asset-0 scale. */
double orc_basket_level_f(const mcq_model* m, const mcq_payoff* p, int n_fine, int M, const double* z,
                          double* yc, double* dd, int flags) {
    int n = m->n_assets, coarse = M > 0, Mr = coarse ? M : 1;
    int dup = m->kind == MCQ_MODEL_MULTI_DUPIRE, own = (flags & MCQ_FLAG_BASKET_OWN_S0) != 0;
    int n_coarse = coarse ? n_fine / Mr : 0;
    double hf = m->T / n_fine, hc = m->T / (n_coarse > 0 ? n_coarse : 1), sq = sqrt(hf);
    double *Sf = (double*)malloc(sizeof(double) * 4 * n), *Sc = Sf + n, *dw = Sf + 2 * n, *acc = Sf + 3 * n;
    for (int a = 0; a < n; a++) { Sf[a] = Sc[a] = m->S0_vec[a]; acc[a] = 0; }
    int unc = m->uncorrelated || !m->L;
    for (int k = 0; k < n_fine; k++) {
        for (int a = 0; a < n; a++) {
            double v = 0;
            if (unc) v = z[k * n + a] * sq;
            else for (int j = 0; j <= a; j++) v += m->L[a * n + j] * z[k * n + j] * sq;
            dw[a] = v;
        }
        for (int a = 0; a < n; a++) {
            double vol = m->sigma_vec ? m->sigma_vec[a] : 0.0;
            if (dup)
                vol = m->sigma0 * exp(-m->alpha * (k * hf)) *
                      pow(Sf[a] / m->S0_vec[own ? a : 0], m->beta_d - 1.0);
            Sf[a] = Sf[a] + m->mu * Sf[a] * hf + vol * Sf[a] * dw[a];
            acc[a] += dw[a];
        }
        if (coarse && (k + 1) % Mr == 0) {
            int kc = (k + 1) / Mr - 1;
            for (int a = 0; a < n; a++) {
                double vol = m->sigma_vec ? m->sigma_vec[a] : 0.0;
                if (dup)
                    vol = m->sigma0 * exp(-m->alpha * (kc * hc)) *
                          pow(Sc[a] / m->S0_vec[own ? a : 0], m->beta_d - 1.0);
                Sc[a] = Sc[a] + m->mu * Sc[a] * hc + vol * Sc[a] * acc[a];
                acc[a] = 0;
            }
        }
    }
    double Bf = 0, Bc = 0, disc = pay_discount(p);
    for (int a = 0; a < n; a++) {
        double w = (m->weights && !dup) ? m->weights[a] : 1.0 / n;
        Bf += w * Sf[a];
        Bc += w * Sc[a];
    }
    double yf = fmax(Bf - p->K, 0.0) * disc;
    *yc = n_coarse > 0 ? fmax(Bc - p->K, 0.0) * disc : 0.0;
    double gf = Bf > p->K ? disc : 0.0, gc = (n_coarse > 0 && Bc > p->K) ? disc : 0.0;
    for (int a = 0; a < n; a++) {
        double w = (m->weights && !dup) ? m->weights[a] : 1.0 / n;
        dd[a] = (dup && !own) ? 0.0 : w / m->S0_vec[a] * (gf * Sf[a] - gc * Sc[a]);
    }
    free(Sf);
    return yf;
}

int orc_basket_level_sums(const mcq_model* m, const mcq_payoff* p, int n_fine, int M, uint32_t salt_base,
                          int R, uint32_t offset, int64_t N, int flags, int n_threads, double* sums) {
    int n = m->n_assets, D = n_fine * n, ns = 4 + n;
    if (D > 20000) return -1;
    if ((uint64_t)offset + (uint64_t)N > 0x100000000ull) return -2;
    int nch = (N < ORC_CHUNKS) ? (int)(N > 0 ? N : 1) : ORC_CHUNKS;
    double* part = (double*)calloc((size_t)R * nch * ns, sizeof(double));
    uint32_t* Lv = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)R * D * 33);
    for (int r = 0; r < R; r++)
        for (int dd = 0; dd < D; dd++) {
            uint32_t* w = Lv + ((size_t)r * D + dd) * 33;
            prescramble(salt_base + (uint32_t)r, dd, w, w + 32);
        }
    int nt = n_threads > 0 ? n_threads : orc_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t task = 0; task < (int64_t)R * nch; task++) {
        int r = (int)(task / nch), c = (int)(task % nch);
        int64_t b = N * c / nch, e = N * (c + 1) / nch;
        if (b >= e) continue;
        uint32_t* x = (uint32_t*)malloc(sizeof(uint32_t) * D);
        double* z = (double*)malloc(sizeof(double) * (D + n));
        double* dd = z + D;
        const uint32_t* L = Lv + (size_t)r * D * 33;
        for (int q = 0; q < D; q++) x[q] = scr_direct(L + q * 33, L[q * 33 + 32], offset + (uint32_t)b);
        double* s = part + (size_t)task * ns;
        for (int64_t i = b; i < e; i++) {
            uint32_t idx = offset + (uint32_t)i;
            if (i > b) { int k = __builtin_ctz(idx); for (int q = 0; q < D; q++) x[q] ^= L[q * 33 + k]; }
            for (int q = 0; q < D; q++) z[q] = orc_ppnd16((double)orc_u_of(x[q], flags));
            double yc, yf = orc_basket_level_f(m, p, n_fine, M, z, &yc, dd, flags);
            double dy = yf - yc;
            s[0] += dy; s[1] += dy * dy; s[2] += yf; s[3] += yf * yf;
            for (int a = 0; a < n; a++) s[4 + a] += dd[a];
        }
        free(x); free(z);
    }
    for (int r = 0; r < R; r++)
        for (int q = 0; q < ns; q++) {
            double a = 0;
            for (int c = 0; c < nch; c++) a += part[((size_t)r * nch + c) * ns + q];
            sums[r * ns + q] = a;
        }
    free(part); free(Lv);
    return 0;
}

int orc_mc_sums(const mcq_model* m, const mcq_payoff* p, int n_steps, uint32_t seed,
                uint32_t stream, int64_t first_path, int64_t n_paths, int n_threads,
                double* sums) {
    int D = n_steps * orc_noise_dim(m);
    int nch = (n_paths < ORC_CHUNKS) ? (int)(n_paths > 0 ? n_paths : 1) : ORC_CHUNKS;
    double* part = (double*)calloc((size_t)nch * 2, sizeof(double));
    int nt = n_threads > 0 ? n_threads : orc_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int c = 0; c < nch; c++) {
        int64_t b = n_paths * c / nch, e = n_paths * (c + 1) / nch;
        double* z = (double*)malloc(sizeof(double) * (D + 4));
        double s1 = 0, s2 = 0;
        for (int64_t i = b; i < e; i++) {
            orc_philox_normals(seed, stream, (uint64_t)(first_path + i), D, z);
            double y = orc_path_payoff(m, p, n_steps, NULL, z);
            s1 += y; s2 += y * y;
        }
        part[c * 2] = s1; part[c * 2 + 1] = s2;
        free(z);
    }
    sums[0] = sums[1] = 0;
    for (int c = 0; c < nch; c++) { sums[0] += part[c * 2]; sums[1] += part[c * 2 + 1]; }
    free(part);
    return 0;
}

/* kernel_is_gbm (methods_cuda.cu:685-707) in FP64: one GBM European path under the drift-shifted
 * measure Z' = Z + z*, with the likelihood ratio exp(-z* sum Z - n z*^2 / 2); z_star is the
 * per-step shift the kernel reads (run_is_cuda passes z_star / sqrt(n_steps), :2297). */
double orc_is_payoff(const mcq_model* m, const mcq_payoff* p, int n_steps, double z_star, const double* z) {
    double h = m->T / n_steps, sh = sqrt(h), S = m->S0, zs = 0.0;
    for (int k = 0; k < n_steps; k++) {
        zs += z[k];
        double dw = (z[k] + z_star) * sh;
        S = S + m->mu * S * h + m->sigma * S * dw;
    }
    double lr = exp(-z_star * zs - 0.5 * z_star * z_star * n_steps);
    return fmax(S - p->K, 0.0) * pay_discount(p) * lr;
}

/* IS sums {sum Y, sum Y^2} per replica: scrambled Sobol (salts salt_base + r, points offset ..
 * offset + N - 1) or Philox (key seed, stream salt_base + r, paths offset ..). */
int orc_is_sums(const mcq_model* m, const mcq_payoff* p, int n_steps, double z_star, int use_sobol,
                uint32_t seed, uint32_t salt_base, int R, uint32_t offset, int64_t N, int flags,
                int n_threads, double* sums) {
    int D = n_steps;
    if (use_sobol && D > 20000) return -1;
    if (use_sobol && (uint64_t)offset + (uint64_t)N > 0x100000000ull) return -2;
    int nch = (N < ORC_CHUNKS) ? (int)(N > 0 ? N : 1) : ORC_CHUNKS;
    double* part = (double*)calloc((size_t)R * nch * 2, sizeof(double));
    uint32_t* Lv = NULL;
    if (use_sobol) {
        Lv = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)R * D * 33);
        for (int r = 0; r < R; r++)
            for (int dd = 0; dd < D; dd++) {
                uint32_t* w = Lv + ((size_t)r * D + dd) * 33;
                prescramble(salt_base + (uint32_t)r, dd, w, w + 32);
            }
    }
    int nt = n_threads > 0 ? n_threads : orc_max_threads();
    (void)nt;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t task = 0; task < (int64_t)R * nch; task++) {
        int r = (int)(task / nch), c = (int)(task % nch);
        int64_t b = N * c / nch, e = N * (c + 1) / nch;
        if (b >= e) continue;
        uint32_t* x = (uint32_t*)malloc(sizeof(uint32_t) * D);
        double* z = (double*)malloc(sizeof(double) * (D + 4));
        const uint32_t* L = use_sobol ? Lv + (size_t)r * D * 33 : NULL;
        if (use_sobol)
            for (int dd = 0; dd < D; dd++) x[dd] = scr_direct(L + dd * 33, L[dd * 33 + 32], offset + (uint32_t)b);
        double s1 = 0, s2 = 0;
        for (int64_t i = b; i < e; i++) {
            if (use_sobol) {
                uint32_t idx = offset + (uint32_t)i;
                if (i > b) {
                    int k = __builtin_ctz(idx);
                    for (int dd = 0; dd < D; dd++) x[dd] ^= L[dd * 33 + k];
                }
                for (int dd = 0; dd < D; dd++) z[dd] = orc_ppnd16((double)orc_u_of(x[dd], flags));
            } else {
                orc_philox_normals(seed, salt_base + (uint32_t)r, (uint64_t)offset + (uint64_t)i, D, z);
            }
            double y = orc_is_payoff(m, p, n_steps, z_star, z);
            s1 += y; s2 += y * y;
        }
        part[task * 2] = s1; part[task * 2 + 1] = s2;
        free(x); free(z);
    }
    for (int r = 0; r < R; r++) {
        double a = 0, b2 = 0;
        for (int c = 0; c < nch; c++) { a += part[((size_t)r * nch + c) * 2]; b2 += part[((size_t)r * nch + c) * 2 + 1]; }
        sums[r * 2] = a; sums[r * 2 + 1] = b2;
    }
    free(part); free(Lv);
    return 0;
}

/* run_qmc_cuda's doubling loop (methods_cuda.cu:1624-1668) with an explicit start size. */
int orc_run_qmc(const mcq_model* m, const mcq_payoff* p, double eps, int n_steps,
                const orc_noise* nz, int R, int max_doublings, int64_t N0, uint32_t salt_base,
                int flags, int n_threads, mcq_result* out) {
    double* acc = (double*)calloc((size_t)R * 2, sizeof(double));
    double* tmp = (double*)calloc((size_t)R * 2, sizeof(double));
    int64_t Nper = N0, Ndone = 0;
    double vom = 1e30, gm = 0, ps = 0;
    int64_t total = 0;
    for (int dbl = 0; dbl < max_doublings; dbl++) {
        if (Nper > 0xFFFFFFFFll) { free(acc); free(tmp); return -2; }
        if (Nper > Ndone) {
            int rc = orc_qmc_sums(m, p, n_steps, nz, salt_base, R, (uint32_t)Ndone, Nper - Ndone,
                                  flags, n_threads, tmp);
            if (rc) { free(acc); free(tmp); return rc; }
            for (int i = 0; i < 2 * R; i++) acc[i] += tmp[i];
            ps += (double)R * (double)(Nper - Ndone) * n_steps;
            Ndone = Nper;
        }
        double mm = 0, v = 0;
        for (int r = 0; r < R; r++) mm += acc[2 * r] / (double)Nper;
        mm /= R;
        for (int r = 0; r < R; r++) { double q = acc[2 * r] / (double)Nper - mm; v += q * q; }
        v = (R > 1) ? v / (R - 1) : 0.0;
        vom = v / R; gm = mm; total = (int64_t)R * Nper;
        if (vom < eps * eps / 2.0) break;
        Nper *= 2;
    }
    out->price = gm; out->std_error = sqrt(vom); out->n_samples = total;
    out->time_s = 0; out->path_steps = ps; out->levels = 1; out->launches = 0;
    free(acc); free(tmp);
    return 0;
}
