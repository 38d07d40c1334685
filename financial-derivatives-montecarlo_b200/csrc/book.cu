// book.cu — a heterogeneous book of correlated GBM basket calls priced by MLQMC with the
// pathwise delta per asset.  No counterpart in the reference, which rejects basket MLQMC
// (methods_cuda.cu:1695-1697) and launches one option at a time with a stream per level
// (:1745-1755).
//
// Each adaptive round collects, for every option still running, the (level, point range)
// slices its MLQMC state machine needs next: the pilots, the optimal extra samples, the pilot
// of a new level (the arithmetic of run_mlqmc_cuda, :1950-2000).  A slice covers all R
// replicas (salts salt_base + l R + r, shared offsets) and is cut into chunks whose size
// depends on the slice alone.  A persistent work-queue kernel per basket-width class (d in 1-4,
// 5-8, 9-12, 13-16, each compiled for its own register budget and specialised on the exact d)
// pulls chunks of every option and level from an atomic counter; k_book_fin turns the chunk
// records of each slice into {mean of the replica means of dY, their sample variance, per-asset
// mean delta}.  The round's kernels are captured once in a CUDA graph and replayed with each
// round's slice list (the counts are read on the device).
//
// The plain comparator runs the same kernels one option at a time, one launch per level on
// that level's own stream — the reference's launch structure.  Chunk records depend only on
// the slice, and each slice is reduced in a fixed order, so both modes give bit-identical
// per-option results.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "book.h"
#include "path_kernels.cuh"
#include "support.h"

namespace mcq {

constexpr int kBookNST = 4 + kMaxBasket;   // per-path statistics in a chunk record
constexpr int kBookOut = 2 + kMaxBasket;   // per slice: E dY, var of replica means, deltas
constexpr int kBookMaxLevels = 12;
constexpr int kBookMaxR = 32;
constexpr int kBookClasses = 5;            // basket width 1-4, 5-8, 9-12, 13-16; single-asset options
constexpr int kSingleClass = 4;
constexpr int kChunkNormals = 8192;        // normals per lane a chunk aims at
constexpr int kMinChunksPerRep = 64;
constexpr int kMaxChunksPerRep = 1024;

// hdr (int32): [0] n_specs, [1] n_chunks, [kHdrChunk0 + c] first chunk of class c (and, at
// c = kBookClasses, n_chunks), [kHdrSlice0 + c] first slice of class c (n_specs at the end),
// [kHdrCounter0 + c] work-queue counter of class c.
constexpr int kHdrChunk0 = 2;
constexpr int kHdrSlice0 = kHdrChunk0 + kBookClasses + 1;
constexpr int kHdrCounter0 = kHdrSlice0 + kBookClasses + 1;
constexpr int kHdrInts = kHdrCounter0 + kBookClasses;

struct BookOptDev {
    double T;
    float K, disc, mu;
    int d, bsk_off, uncorrelated;
    int kp;   // single-asset option: its level-0 parameter block in BookArgs::kps (level l at kp + l); -1: basket
};

struct BookSpec {   // one (option, level) slice: all replicas, points [offset, offset + n_points)
    int opt, level;
    uint32_t offset, n_points;
    int gpc, cpr, chunk0, pad;
};

struct BookArgs {
    int* hdr;
    const BookSpec* specs;
    const BookOptDev* opts;
    const float* bdata;   // per option [S0 | sigma | weight | L (d x d row-major)]
    const KParams* kps;   // single-asset options: one fused-pass parameter block per (option, level)
    const uint32_t* dirs[kBookMaxLevels];
    int dstride[kBookMaxLevels];
    int R, M, n0;
    float u_cap;
    double* records;      // [chunk][kBookNST]
    double* out;          // [slice][kBookOut]
};

__host__ __device__ inline int book_class(int d) { return (d - 1) >> 2; }

// Per-warp shared memory: the 32 x 32 transpose tile, the option's Cholesky factor with rows
// padded to a multiple of 4 floats, its per-asset constants (sigma, S0, weight, weight / S0), and
// the FP64 record of the chunk.
constexpr int kBookLsFloats = kMaxBasket * kMaxBasket;
constexpr int kBookAssetFloats = 4 * kMaxBasket;   // sigma, S0, weight, weight / S0 per asset
constexpr int kBookWarpFloats = 1024 + kBookLsFloats + kBookAssetFloats + 2 * kBookNST;
// Baskets of 11 and 12 assets leave many lanes of a step-major tile idle (a 32-dimension tile holds
// 22 or 24 whole-step dimensions); they generate two tiles at a time instead, holding 64 / d whole
// steps (55 or 60 of 64 lanes busy): 1.08-1.17x on their slices.  Their class (d 9-12) gets a second
// transpose tile after the per-warp area.  Pairing gained nothing at d = 9 and cost 4-7 % in the
// d 5-8 class (d = 7, and d = 8 through the larger kernel), so those keep single tiles.
__host__ __device__ constexpr bool book_pair_tiles(int d) { return d == 11 || d == 12; }
// After them, the Sobol start words a warp carries from group to group of a chunk (sobol_tile): one
// 32-word slot per tile for a path's first kBookCarryTiles tiles (a chunk's later tiles walk their
// start word), sized so that the basket classes keep three resident CTAs per SM; the single-asset
// class carries paths of up to kBookSingleCarryTiles tiles whole.
constexpr int kBookCarryTiles = 24;
constexpr int kBookSingleCarryTiles = 16;
__host__ __device__ constexpr int book_warp_floats(int cls) {
    return kBookWarpFloats + (cls == 2 ? 1024 : 0) + 32 * kBookCarryTiles;
}
constexpr int kBookSingleWarpFloats = 1024 + 32 * kBookSingleCarryTiles;

// A float4 of shared memory, read at every use.  The Cholesky rows are loop-invariant and the
// compiler otherwise keeps the factor in registers across the chunk; for baskets of up to four
// assets, reading it at every step lets the class run at 64 registers (four CTAs per SM instead
// of three: 1.08-1.17x).  The wider classes keep the cached factor (re-reading it and a
// tighter budget made d = 5-8 3-7 % slower and d = 9-12 no faster).
__device__ __forceinline__ float4 lds4(const float4* p) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"((unsigned)__cvta_generic_to_shared(p)));
    return v;
}

// The coupled basket pair of one path for a basket of exactly D assets: the correlated Euler
// step S + S (mu h + sigma dW) with dW = L x, x = z sqrt(h), coarse steps on the summed fine
// increments every M fine steps, the call on the weighted basket and d payoff / d S0_a =
// disc 1{B > K} w_a S_a(T) / S0_a.  Same operations in the same order as the fused pass's
// coupled basket consumer, so a slice gives the values the single-option MLQMC driver gives.
template <int D>
struct BookPath {
    static constexpr int DP = (D + 3) & ~3, NS = 4 + D;
    float Sf[D], Sc[D], acc[D];
    int m;
    // as: the per-asset constants in shared memory, [sigma | S0 | weight | weight / S0]
    __device__ __forceinline__ void init(const float* as) {
#pragma unroll
        for (int q = 0; q < D; q++) {
            Sf[q] = Sc[q] = as[kMaxBasket + q];
            acc[q] = 0.f;
        }
        m = 0;
    }
    // x: this step's D normals times sqrt(h); L4: lower Cholesky rows padded to DP floats
    __device__ __forceinline__ void step(const float (&x)[D], const float4* L4, const float* sg, float muh_f,
                                         float muh_c, int Mc) {
#pragma unroll
        for (int q = 0; q < D; q++) {
            float dw = 0.f;
#pragma unroll
            for (int j4 = 0; j4 <= q / 4; j4++) {
                const float4 v = (D <= 4) ? lds4(L4 + (q * DP) / 4 + j4) : L4[(q * DP) / 4 + j4];
                dw = fmaf(v.x, x[4 * j4], dw);
                if (4 * j4 + 1 <= q) dw = fmaf(v.y, x[4 * j4 + 1], dw);
                if (4 * j4 + 2 <= q) dw = fmaf(v.z, x[4 * j4 + 2], dw);
                if (4 * j4 + 3 <= q) dw = fmaf(v.w, x[4 * j4 + 3], dw);
            }
            Sf[q] = fmaf(Sf[q], fmaf(sg[q], dw, muh_f), Sf[q]);
            acc[q] += dw;
        }
        if (++m == Mc) {
#pragma unroll
            for (int q = 0; q < D; q++) {
                Sc[q] = fmaf(Sc[q], fmaf(sg[q], acc[q], muh_c), Sc[q]);
                acc[q] = 0.f;
            }
            m = 0;
        }
    }
    __device__ __forceinline__ void finish(const float* as, float K, float disc, bool has_c, float (&y)[NS]) const {
        float Bf = 0.f, Bc = 0.f;
#pragma unroll
        for (int q = 0; q < D; q++) {
            const float w = as[2 * kMaxBasket + q];
            Bf = fmaf(w, Sf[q], Bf);
            Bc = fmaf(w, Sc[q], Bc);
        }
        const float yf = fmaxf(Bf - K, 0.f) * disc;
        const float yc = has_c ? fmaxf(Bc - K, 0.f) * disc : 0.f;
        const float dy = yf - yc;
        const float gf = (Bf > K) ? disc : 0.f, gc = (has_c && Bc > K) ? disc : 0.f;
        y[0] = dy; y[1] = dy * dy; y[2] = yf; y[3] = yf * yf;
#pragma unroll
        for (int q = 0; q < D; q++) {
            y[4 + q] = as[3 * kMaxBasket + q] * (gf * Sf[q] - gc * Sc[q]);   // w_a / S0_a, staged per chunk
        }
    }
};

// Chunk accumulator of the per-path statistics.  Narrow baskets (NS <= 12) keep FP64 sums per
// lane and reduce across the warp once per chunk: their paths are short, and a warp reduction
// per path would cost as much as the path.  Wider ones add each path's warp sum (FP32 shuffle
// tree) to an FP64 record in shared memory, keeping their registers for the path state.
template <int NS, bool LANE = (NS <= 12)>
struct BookAcc {
    double v[LANE ? NS : 1];
    double* wrec;
    __device__ __forceinline__ void init(double* w, int lane) {
        wrec = w;
        if constexpr (LANE) {
#pragma unroll
            for (int q = 0; q < NS; q++) v[q] = 0.0;
        } else {
            if (lane < NS) wrec[lane] = 0.0;
            __syncwarp();
        }
    }
    __device__ __forceinline__ void add(const float (&y)[NS], bool valid, int lane) {
        if constexpr (LANE) {
            if (valid) {
#pragma unroll
                for (int q = 0; q < NS; q++) v[q] += (double)y[q];
            }
        } else {
#pragma unroll
            for (int q = 0; q < NS; q++) {
                float t = valid ? y[q] : 0.f;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
                if (lane == 0) wrec[q] += (double)t;
            }
        }
    }
    // writes the chunk record [kBookNST] (zeros past NS)
    __device__ __forceinline__ void flush(double* rec, int lane) {
        if constexpr (LANE) {
#pragma unroll
            for (int q = 0; q < NS; q++) {
                double t = v[q];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
                v[q] = t;
            }
            if (lane < kBookNST) {
                double out = 0.0;
#pragma unroll
                for (int q = 0; q < NS; q++)
                    if (lane == q) out = v[q];
                rec[lane] = out;
            }
        } else {
            __syncwarp();
            if (lane < kBookNST) rec[lane] = (lane < NS) ? wrec[lane] : 0.0;
        }
        __syncwarp();
    }
};

// One chunk of a slice for a basket of exactly D assets: groups [gb, ge) of replica r.
//
// Paths of Dt = nf D <= 16 normals (the low levels of baskets of up to 8 assets) take
// Q = 32 / Dt groups per Sobol tile: lane j generates dimension j mod Dt of group g + j / Dt,
// and each lane then steps its Q paths from the transposed tile.  Longer paths are generated
// step-major: a tile holds S = 32 / D whole steps (W = S D dimensions, lane j < W owning
// dimension k0 D + j), so every normal of a step sits in known registers after the transpose
// and L x is an unrolled triangular product with L read as float4 broadcasts.
template <int D>
__device__ __forceinline__ void book_chunk(const BookArgs& a, const BookSpec& s, const BookOptDev& o, int r,
                                           uint64_t gb, uint64_t ge, float* buf, float* Ls, double* wrec,
                                           double* rec, uint32_t* carry, int lane) {
    using P = BookPath<D>;
    constexpr int S = 32 / D, W = S * D, DP = P::DP, NS = P::NS;
    const float* bk = a.bdata + o.bsk_off;
    for (int i = lane; i < D * DP; i += 32) {
        const int row = i / DP, col = i - row * DP;
        Ls[i] = (col <= row) ? __ldg(bk + 3 * D + row * D + col) : 0.f;
    }
    BookAcc<NS> acc;
    acc.init(wrec, lane);
    float* sg = Ls + kBookLsFloats;   // per-asset constants: sigma (read at every step), S0, w, w / S0
    if (lane < D) {
        const float s0 = __ldg(bk + lane), w = __ldg(bk + 2 * D + lane);
        sg[lane] = __ldg(bk + D + lane);
        sg[kMaxBasket + lane] = s0;
        sg[2 * kMaxBasket + lane] = w;
        sg[3 * kMaxBasket + lane] = w / s0;
    }
    int nf = a.n0;
    for (int l = 0; l < s.level; l++) nf *= a.M;
    const int nc = s.level ? nf / a.M : 0;
    const int Mc = s.level ? a.M : INT_MAX;   // the coarse path never steps on level 0
    const float h = (float)(o.T / nf);
    const float sqrt_h = sqrtf(h);
    const float hc = (float)(o.T / max(nc, 1));
    const float muh_f = o.mu * h, muh_c = o.mu * hc;
    const float K = o.K, disc = o.disc;
    const bool has_c = nc > 0;
    const int dstride = a.dstride[s.level];
    const uint32_t* dr = a.dirs[s.level] + (size_t)r * 33 * (size_t)dstride;
    const int Dt = nf * D;
    const uint64_t pend = (uint64_t)s.offset + s.n_points;
    const float4* L4 = reinterpret_cast<const float4*>(Ls);
    __syncwarp();
    if (D <= 8 && 2 * Dt <= 32) {   // wider baskets keep their registers for the step-major path
        const int Q = 32 / Dt, qj = lane / Dt, dj = lane - qj * Dt;
        for (uint64_t g = gb; g < ge; g += Q) {
            const uint64_t gl = g + (uint64_t)qj;
            sobol_tile(dr, dstride, dj, qj < Q && gl < ge, gl, a.u_cap, buf, lane);
            __syncwarp();
            for (int q = 0; q < Q && g + q < ge; q++) {
                P path;
                path.init(sg);
                for (int k = 0; k < nf; k++) {
                    float x[D];
#pragma unroll
                    for (int c = 0; c < D; c++) x[c] = buf[swz(lane, q * Dt + k * D + c)] * sqrt_h;
                    path.step(x, L4, sg, muh_f, muh_c, Mc);
                }
                float y[NS];
                path.finish(sg, K, disc, has_c, y);
                const uint64_t n = (g + q) * 32 + (uint64_t)lane;
                acc.add(y, n >= s.offset && n < pend, lane);
            }
            __syncwarp();
        }
    } else if constexpr (book_pair_tiles(D)) {
        // two tiles per round: dimensions k0 D .. k0 D + 63, S2 = 64 / D whole steps
        constexpr int S2 = 64 / D, W2 = S2 * D;
        float* buf2 = buf + kBookWarpFloats;
        for (uint64_t g = gb; g < ge; g++) {
            P path;
            path.init(sg);
            for (int k0 = 0, t = 0; k0 < nf; k0 += S2, t += 2) {
                const int dim = k0 * D + lane;
                const bool cont = g != gb;
                sobol_tile(dr, dstride, dim, dim < Dt, g, a.u_cap, buf, lane,
                           t < kBookCarryTiles ? carry + 32 * t + lane : nullptr, cont);
                sobol_tile(dr, dstride, dim + 32, lane < W2 - 32 && dim + 32 < Dt, g, a.u_cap, buf2, lane,
                           t + 1 < kBookCarryTiles ? carry + 32 * (t + 1) + lane : nullptr, cont);
                __syncwarp();
                const float4* rowA = reinterpret_cast<const float4*>(buf + lane * 32);
                const float4* rowB = reinterpret_cast<const float4*>(buf2 + lane * 32);
#pragma unroll
                for (int st = 0; st < S2; st++) {
                    if (k0 + st < nf) {
                        float x[D];
#pragma unroll
                        for (int c = 0; c < D; c++) {
                            const int col = st * D + c;
                            const float4 v = (col < 32) ? rowA[(col >> 2) ^ (lane & 7)]
                                                        : rowB[((col - 32) >> 2) ^ (lane & 7)];
                            const float zc = (col & 3) == 0 ? v.x : (col & 3) == 1 ? v.y : (col & 3) == 2 ? v.z : v.w;
                            x[c] = zc * sqrt_h;
                        }
                        path.step(x, L4, sg, muh_f, muh_c, Mc);
                    }
                }
                __syncwarp();
            }
            float y[NS];
            path.finish(sg, K, disc, has_c, y);
            const uint64_t n = g * 32 + (uint64_t)lane;
            acc.add(y, n >= s.offset && n < pend, lane);
        }
    } else {
        for (uint64_t g = gb; g < ge; g++) {
            P path;
            path.init(sg);
            for (int k0 = 0, t = 0; k0 < nf; k0 += S, t++) {
                const int dim = k0 * D + lane;
                sobol_tile(dr, dstride, dim, lane < W && dim < Dt, g, a.u_cap, buf, lane,
                           t < kBookCarryTiles ? carry + 32 * t + lane : nullptr, g != gb);
                __syncwarp();
                // this path's row of the tile, read per step as float4 chunks (conflict-free in
                // the swizzled layout) so that only one step's normals are live in registers
                const float4* row4 = reinterpret_cast<const float4*>(buf + lane * 32);
#pragma unroll
                for (int st = 0; st < S; st++) {
                    if (k0 + st < nf) {
                        float x[D];
#pragma unroll
                        for (int c = 0; c < D; c++) {
                            const int col = st * D + c;
                            const float4 v = row4[(col >> 2) ^ (lane & 7)];
                            const float zc = (col & 3) == 0 ? v.x : (col & 3) == 1 ? v.y : (col & 3) == 2 ? v.z : v.w;
                            x[c] = zc * sqrt_h;
                        }
                        path.step(x, L4, sg, muh_f, muh_c, Mc);
                    }
                }
                __syncwarp();
            }
            float y[NS];
            path.finish(sg, K, disc, has_c, y);
            const uint64_t n = g * 32 + (uint64_t)lane;
            acc.add(y, n >= s.offset && n < pend, lane);
        }
    }
    acc.flush(rec, lane);
}

// Persistent work-queue kernel of one width class: warps take chunks from the class's atomic
// counter until the round's chunks run out.
template <int CLS, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) k_book(const __grid_constant__ BookArgs a) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    float* buf = reinterpret_cast<float*>(smem4) + wib * book_warp_floats(CLS);
    uint32_t* carry = reinterpret_cast<uint32_t*>(buf + book_warp_floats(CLS) - 32 * kBookCarryTiles);
    float* Ls = buf + 1024;
    double* wrec = reinterpret_cast<double*>(Ls + kBookLsFloats + kBookAssetFloats);
    const int c_end = a.hdr[kHdrChunk0 + CLS + 1];
    const int s_beg = a.hdr[kHdrSlice0 + CLS], s_last = a.hdr[kHdrSlice0 + CLS + 1] - 1;
    for (;;) {
        int c = 0;
        if (lane == 0) c = a.hdr[kHdrChunk0 + CLS] + atomicAdd(a.hdr + kHdrCounter0 + CLS, 1);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= c_end) break;
        int lo = s_beg, hi = s_last;   // last slice of the class with chunk0 <= c
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.specs[mid].chunk0 <= c) lo = mid; else hi = mid - 1;
        }
        const BookSpec s = a.specs[lo];
        const BookOptDev o = a.opts[s.opt];
        const int q = c - s.chunk0, r = q / s.cpr, j = q - r * s.cpr;
        const uint64_t gend = ((uint64_t)s.offset + s.n_points - 1) / 32 + 1;
        const uint64_t gb = (s.offset >> 5) + (uint64_t)j * (uint64_t)s.gpc;
        const uint64_t ge = min(gb + (uint64_t)s.gpc, gend);
        double* rec = a.records + (size_t)c * kBookNST;
        switch (o.d - 4 * CLS) {
            case 1: book_chunk<4 * CLS + 1>(a, s, o, r, gb, ge, buf, Ls, wrec, rec, carry, lane); break;
            case 2: book_chunk<4 * CLS + 2>(a, s, o, r, gb, ge, buf, Ls, wrec, rec, carry, lane); break;
            case 3: book_chunk<4 * CLS + 3>(a, s, o, r, gb, ge, buf, Ls, wrec, rec, carry, lane); break;
            default: book_chunk<4 * CLS + 4>(a, s, o, r, gb, ge, buf, Ls, wrec, rec, carry, lane); break;
        }
    }
}

// One chunk of a single-asset option's slice: the fused pass's coupled fine / coarse consumer
// (PathC, the pair mcq_run_mlqmc prices) on raw scrambled-Sobol normals, groups [gb, ge) of
// replica r, with the option's parameter block for the slice's level.  Record: {dY, dY^2, Yf,
// Yf^2} and zeros in place of the basket deltas.
template <class C>
__device__ __forceinline__ void single_chunk(const KParams& kp, const BookSpec& s, int r, uint64_t gb, uint64_t ge,
                                             const uint32_t* dr, float* buf, double* rec, int lane) {
    Acc<C::NST> acc;
    acc.zero();
    const uint64_t pend = (uint64_t)s.offset + s.n_points;
    uint32_t* carry = ((kp.D + 31) / 32 <= kBookSingleCarryTiles) ? reinterpret_cast<uint32_t*>(buf + 1024) : nullptr;
    for (uint64_t h = gb; h < ge; h++) {
        const uint64_t n = h * 32 + (uint64_t)lane;
        C cons;
        cons.init(kp);
        cons.bind(r, n);
        run_group<GEN_SOBOL, NOISE_RAW>(kp, cons, dr, 0u, h, n, buf, nullptr, lane, carry, h != gb);
        float y[C::NST];
        cons.finish(kp, y);
        if (n >= s.offset && n < pend) acc.add(y);
    }
    acc.flush(rec, lane);
    for (int q = C::NST + lane; q < kBookNST; q += 32) rec[q] = 0.0;
}

template <int MOD>
__device__ __forceinline__ void single_chunk_pay(const KParams& kp, const BookSpec& s, int r, uint64_t gb,
                                                 uint64_t ge, const uint32_t* dr, float* buf, double* rec, int lane) {
    switch (kp.payoff) {
        case PAY_ASIAN: single_chunk<PathC<MOD, PAY_ASIAN, true>>(kp, s, r, gb, ge, dr, buf, rec, lane); break;
        case PAY_GEOM: single_chunk<PathC<MOD, PAY_GEOM, true>>(kp, s, r, gb, ge, dr, buf, rec, lane); break;
        case PAY_LOOKBACK: single_chunk<PathC<MOD, PAY_LOOKBACK, true>>(kp, s, r, gb, ge, dr, buf, rec, lane); break;
        case PAY_UPOUT: single_chunk<PathC<MOD, PAY_UPOUT, true>>(kp, s, r, gb, ge, dr, buf, rec, lane); break;
        case PAY_DOWNOUT: single_chunk<PathC<MOD, PAY_DOWNOUT, true>>(kp, s, r, gb, ge, dr, buf, rec, lane); break;
        default: single_chunk<PathC<MOD, PAY_EUR, true>>(kp, s, r, gb, ge, dr, buf, rec, lane); break;
    }
}

// Persistent work-queue kernel of the single-asset class: warps take chunks of every such option and
// level from the class's counter; each chunk runs its option's model and payoff.
template <int MINB>
__global__ void __launch_bounds__(kThreads, MINB) k_book_single(const __grid_constant__ BookArgs a) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    float* buf = reinterpret_cast<float*>(smem4) + wib * kBookSingleWarpFloats;
    const int c_end = a.hdr[kHdrChunk0 + kSingleClass + 1];
    const int s_beg = a.hdr[kHdrSlice0 + kSingleClass], s_last = a.hdr[kHdrSlice0 + kSingleClass + 1] - 1;
    for (;;) {
        int c = 0;
        if (lane == 0) c = a.hdr[kHdrChunk0 + kSingleClass] + atomicAdd(a.hdr + kHdrCounter0 + kSingleClass, 1);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= c_end) break;
        int lo = s_beg, hi = s_last;   // last slice of the class with chunk0 <= c
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.specs[mid].chunk0 <= c) lo = mid; else hi = mid - 1;
        }
        const BookSpec s = a.specs[lo];
        const KParams& kp = a.kps[a.opts[s.opt].kp + s.level];
        const int q = c - s.chunk0, r = q / s.cpr, j = q - r * s.cpr;
        const uint64_t gend = ((uint64_t)s.offset + s.n_points - 1) / 32 + 1;
        const uint64_t gb = (s.offset >> 5) + (uint64_t)j * (uint64_t)s.gpc;
        const uint64_t ge = min(gb + (uint64_t)s.gpc, gend);
        const uint32_t* dr = a.dirs[s.level] + (size_t)r * 33 * (size_t)a.dstride[s.level];
        double* rec = a.records + (size_t)c * kBookNST;
        switch (kp.model) {
            case MOD_HESTON: single_chunk_pay<MOD_HESTON>(kp, s, r, gb, ge, dr, buf, rec, lane); break;
            case MOD_DUPIRE: single_chunk_pay<MOD_DUPIRE>(kp, s, r, gb, ge, dr, buf, rec, lane); break;
            default: single_chunk_pay<MOD_GBM>(kp, s, r, gb, ge, dr, buf, rec, lane); break;
        }
    }
}

// Per slice: the replica sums of its chunk records, then the mean of the replica means of dY,
// their sample variance and the mean per-asset delta.  One CTA per slice and one warp per
// replica: lane l adds the records of chunks l, l + 32, l + 64, ... in that order, the 32 lane
// sums are combined by an xor butterfly (offsets 16, 8, 4, 2, 1), and warp 0 forms the slice
// statistics from the R replica sums in replica order.  book_level_sums restates the same
// order on the host.
constexpr int kFinStats = 1 + kMaxBasket;   // dY and the deltas: record entries 0 and 4 ..
__global__ void k_book_fin(const __grid_constant__ BookArgs a) {
    __shared__ double rs[kBookMaxR][kFinStats];
    const int lane = threadIdx.x & 31, rw = threadIdx.x >> 5;
    const int n_specs = a.hdr[0];
    for (int s = blockIdx.x; s < n_specs; s += gridDim.x) {
        const BookSpec sp = a.specs[s];
        if (rw < a.R) {
            double v[kFinStats];
#pragma unroll
            for (int k = 0; k < kFinStats; k++) v[k] = 0.0;
            for (int j = lane; j < sp.cpr; j += 32) {
                const double* rec = a.records + (size_t)(sp.chunk0 + rw * sp.cpr + j) * kBookNST;
                v[0] += rec[0];
#pragma unroll
                for (int k = 1; k < kFinStats; k++) v[k] += rec[3 + k];
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
                for (int k = 0; k < kFinStats; k++) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
            }
            if (lane == 0) {
#pragma unroll
                for (int k = 0; k < kFinStats; k++) rs[rw][k] = v[k];
            }
        }
        __syncthreads();
        if (rw == 0 && lane < kFinStats) {
            double rep[kBookMaxR];
            double m = 0.0;
            for (int r = 0; r < a.R; r++) {
                rep[r] = rs[r][lane] / (double)sp.n_points;
                m += rep[r];
            }
            m /= a.R;
            double* o = a.out + (size_t)s * kBookOut;
            if (lane == 0) {
                double v = 0.0;
                // separate roundings (no fused multiply-add), so that a host restatement in IEEE
                // double gives the same bits
                for (int r = 0; r < a.R; r++) v = __dadd_rn(v, __dmul_rn(rep[r] - m, rep[r] - m));
                o[0] = m;
                o[1] = a.R > 1 ? v / (a.R - 1) : 0.0;
            } else {
                o[1 + lane] = m;
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ host

void book_validate(const mcq_book_option* opts, int n, const mcq_mlmc_cfg& ml, const mcq_qmc_cfg& qc) {
    MCQ_REQUIRE(opts && n >= 1, MCQ_ERR_INVALID, "book: needs at least one option");
    MCQ_REQUIRE(qc.R >= 2 && qc.R <= kBookMaxR, MCQ_ERR_UNSUPPORTED, "book: R must be 2..32 replicas");
    MCQ_REQUIRE(ml.M >= 2 && ml.n0_steps >= 1 && ml.pilot_n >= 1, MCQ_ERR_INVALID,
                "book: needs M >= 2, n0_steps >= 1, pilot_n >= 1");
    for (int i = 0; i < n; i++) {
        const mcq_book_option& o = opts[i];
        const std::string tag = "book option " + std::to_string(i) + ": ";
        if (o.model) {   // single-asset option
            MCQ_REQUIRE(o.payoff, MCQ_ERR_INVALID, tag + "a model needs a payoff");
            const int mk = o.model->kind, pk = o.payoff->kind;
            MCQ_REQUIRE(mk == MCQ_MODEL_GBM || mk == MCQ_MODEL_HESTON || mk == MCQ_MODEL_DUPIRE, MCQ_ERR_UNSUPPORTED,
                        tag + "single-asset book options take GBM, Heston or parametric Dupire models");
            MCQ_REQUIRE(pk == MCQ_PAYOFF_EUROPEAN || pk == MCQ_PAYOFF_ASIAN || pk == MCQ_PAYOFF_GEOM_ASIAN ||
                            pk == MCQ_PAYOFF_LOOKBACK || pk == MCQ_PAYOFF_BARRIER_UP_OUT ||
                            pk == MCQ_PAYOFF_BARRIER_DOWN_OUT,
                        MCQ_ERR_UNSUPPORTED, tag + "unsupported payoff for a single-asset book option");
            MCQ_REQUIRE(o.max_L >= 2 && o.max_L < kBookMaxLevels, MCQ_ERR_INVALID, tag + "max_L must be 2..11");
            MCQ_REQUIRE(o.eps > 0 && o.model->T > 0, MCQ_ERR_INVALID, tag + "needs eps > 0 and T > 0");
            const long long dn = (mk == MCQ_MODEL_HESTON) ? 2 : 1;
            long long nf = ml.n0_steps;
            for (int l = 0; l < o.max_L && nf <= 20000; l++) nf *= ml.M;
            MCQ_REQUIRE(nf * dn <= 20000, MCQ_ERR_RANGE,
                        tag + "finest level x factors exceeds the 20000 Sobol dimensions of the table");
            continue;
        }
        MCQ_REQUIRE(o.n_assets >= 1 && o.n_assets <= kMaxBasket, MCQ_ERR_UNSUPPORTED, tag + "needs 1..16 assets");
        MCQ_REQUIRE(o.max_L >= 2 && o.max_L < kBookMaxLevels, MCQ_ERR_INVALID, tag + "max_L must be 2..11");
        MCQ_REQUIRE(o.eps > 0 && o.T > 0 && o.S0 && o.sigma, MCQ_ERR_INVALID, tag + "needs eps > 0, T > 0, S0, sigma");
        long long nf = ml.n0_steps;
        for (int l = 0; l < o.max_L && nf <= 20000; l++) nf *= ml.M;
        MCQ_REQUIRE(nf * o.n_assets <= 20000, MCQ_ERR_RANGE,
                    tag + "finest level x assets exceeds the 20000 Sobol dimensions of the table");
    }
}

namespace {

constexpr int kIterCap = 50;   // run_mlqmc_cuda's iteration cap (:1950)

size_t book_smem(int cls) {
    return (size_t)kWarpsPerBlock * (cls == kSingleClass ? kBookSingleWarpFloats : book_warp_floats(cls)) * sizeof(float);
}

// normals a path of the option takes per step (assets of a basket, factors of a single-asset model)
inline int book_width(const mcq_book_option& o) {
    return o.model ? (o.model->kind == MCQ_MODEL_HESTON ? 2 : 1) : o.n_assets;
}
inline int book_class_of(const mcq_book_option& o) { return o.model ? kSingleClass : book_class(o.n_assets); }

// Resident CTAs per SM each width class is compiled for (its register budget): two launch
// variants per class, the measured default and one more CTA per SM (d 1-4: one fewer), which
// differ only in register allocation; the autotuner keeps the faster per class.
using BookFn = void (*)(BookArgs);
constexpr int kBookVariants = 2;
BookFn book_fn(int cls, int variant) {
    switch (cls * kBookVariants + variant) {
        case 0: return k_book<0, 4>;
        case 1: return k_book<0, 3>;
        case 2: return k_book<1, 2>;
        case 3: return k_book<1, 3>;
        case 4: return k_book<2, 2>;
        case 5: return k_book<2, 3>;
        case 6: return k_book<3, 2>;
        case 7: return k_book<3, 3>;
        case 8: return k_book_single<3>;
        default: return k_book_single<4>;
    }
}
inline uint64_t book_tune_key(int cls) { return (2ULL << 40) | (uint64_t)cls; }
// the variant the tuner has settled on for a class (0 while it is still trying)
inline int book_variant(int cls) {
    const TuneState* ts = tune_state(book_tune_key(cls));
    return (ts && ts->chosen >= 0) ? ts->chosen : 0;
}

struct OptState {
    int L = 2, iter = 0, phase = 0;   // phase 0: first pilots, 1: extras, 2: pilot of level L
    bool done = false, converged = false;
    double E[kBookMaxLevels] = {}, sig2[kBookMaxLevels] = {};
    long long N[kBookMaxLevels] = {}, next_off[kBookMaxLevels] = {};
    double Dl[kBookMaxLevels][kMaxBasket] = {};
    int n_pending = 0;
    int pend_level[kBookMaxLevels];
    long long pend_n[kBookMaxLevels];
};

// Grow-only with doubling, so that a book's rounds reallocate (and the batched graph is
// re-captured) a logarithmic number of times.
inline void* grow(DevBuf& b, size_t bytes) { return b.ensure(bytes <= b.cap ? bytes : std::max(bytes, 2 * b.cap)); }

// Device and pinned buffers of one launch context (the batched round, or one level stream):
// the engine workspace's long-lived scratch, so that a book allocates only when it needs more
// than an earlier one (an allocation or free would synchronise the device inside the run).
struct Slot {
    cudaStream_t stream;
    DevBuf &specs, &hdr, &records, &out;
    PinnedBuf &hspecs, &hout;
    explicit Slot(Workspace& w)
        : stream(w.stream), specs(w.xbuf[0]), hdr(w.xbuf[1]), records(w.xbuf[2]), out(w.xbuf[3]),
          hspecs(w.xpin[0]), hout(w.xpin[1]) {}
};

}  // namespace

struct BookRunner {
    const mcq_book_option* opts = nullptr;
    int n = 0;
    mcq_mlmc_cfg ml{};
    mcq_qmc_cfg qc{};
    int R = 0, M = 0, n0 = 0, max_L_all = 2;
    DevBuf* d_opts = nullptr;     // engine scratch (workspace 0)
    DevBuf* d_bdata = nullptr;
    DevBuf* d_kps = nullptr;      // single-asset options' parameter blocks
    std::vector<DevBuf*> dirs;    // level l's table in workspace 1 + l
    std::vector<int> dstride;
    std::vector<OptState> st;
    size_t max_specs = 0;
    long long launches = 0, rounds = 0;
    double path_steps = 0, normals = 0;

    long long nfine(int l) const {
        long long v = n0;
        for (int i = 0; i < l; i++) v *= M;
        return v;
    }

    BookArgs args(Slot& s) const {
        BookArgs a;
        std::memset(&a, 0, sizeof(a));
        a.hdr = (int*)s.hdr.p;
        a.specs = (const BookSpec*)s.specs.p;
        a.opts = (const BookOptDev*)d_opts->p;
        a.bdata = (const float*)d_bdata->p;
        a.kps = (const KParams*)d_kps->p;
        for (int l = 0; l <= max_L_all; l++) {
            a.dirs[l] = (const uint32_t*)dirs[l]->p;
            a.dstride[l] = dstride[l];
        }
        a.R = R; a.M = M; a.n0 = n0;
        a.u_cap = ((qc.flags | ml.flags) & MCQ_FLAG_COMPAT_U_INF) ? 1.0f : 0x1.fffffep-1f;
        a.records = (double*)s.records.p;
        a.out = (double*)s.out.p;
        return a;
    }

    void setup() {
        Engine& E = engine();
        book_validate(opts, n, ml, qc);
        R = qc.R; M = ml.M; n0 = ml.n0_steps;
        std::vector<BookOptDev> ho(n);
        std::vector<float> bd;
        std::vector<KParams> kps;
        int dmax = 1;
        for (int i = 0; i < n; i++) {
            const mcq_book_option& o = opts[i];
            if (o.model) {
                // one fused-pass parameter block per level, as mcq_run_mlqmc fills it for the
                // level's coupled pass (its table stride is the book's, set below)
                ho[i] = BookOptDev{o.model->T, 0.f, 0.f, 0.f, book_width(o), 0, 1, (int)kps.size()};
                for (int l = 0; l < kBookMaxLevels; l++) {
                    KParams k{};
                    if (l <= o.max_L) {
                        PassArgs pa;
                        pa.m = o.model; pa.p = o.payoff; pa.n_steps = (int)nfine(l); pa.est = EST_COUPLED;
                        pa.M = M; pa.level0 = (l == 0); pa.mlmc_h = true; pa.R = R; pa.gen = GEN_SOBOL;
                        pa.noise = NOISE_RAW; pa.flags = ml.flags | qc.flags;
                        Workspace none;   // no staged arrays for these models
                        fill_params(none, pa, k);
                    }
                    kps.push_back(k);
                }
                max_L_all = std::max(max_L_all, o.max_L);
                dmax = std::max(dmax, book_width(o));
                continue;
            }
            const int d = o.n_assets;
            ho[i] = BookOptDev{o.T, (float)o.K, (float)std::exp(-o.r * o.T), (float)o.r, d, (int)bd.size(),
                               o.L ? 0 : 1, -1};
            for (int a = 0; a < d; a++) bd.push_back((float)o.S0[a]);
            for (int a = 0; a < d; a++) bd.push_back((float)o.sigma[a]);
            for (int a = 0; a < d; a++) bd.push_back(o.weights ? (float)o.weights[a] : 1.0f / d);
            for (int a = 0; a < d; a++)
                for (int b = 0; b < d; b++) bd.push_back(o.L ? (float)o.L[a * d + b] : (a == b ? 1.f : 0.f));
            max_L_all = std::max(max_L_all, o.max_L);
            dmax = std::max(dmax, d);
        }
        cudaStream_t s0 = E.ws(0).stream;
        d_opts = &E.ws(0).xbuf[5];
        d_bdata = &E.ws(0).xbuf[6];
        d_kps = &E.ws(0).xbuf[7];
        MCQ_CUDA(cudaMemcpyAsync(grow(*d_opts, sizeof(BookOptDev) * n), ho.data(), sizeof(BookOptDev) * n,
                                 cudaMemcpyHostToDevice, s0));
        MCQ_CUDA(cudaMemcpyAsync(grow(*d_bdata, sizeof(float) * bd.size()), bd.data(), sizeof(float) * bd.size(),
                                 cudaMemcpyHostToDevice, s0));
        // one scrambled table per level shared by all options; an option of d assets uses its
        // first nfine(l) d dimensions, exactly the table run_mlqmc builds for it
        dirs.assign(max_L_all + 1, nullptr);
        dstride.assign(max_L_all + 1, 0);
        for (int l = 0; l <= max_L_all; l++) {
            dstride[l] = (int)(dmax * nfine(l));
            dirs[l] = &E.ws(1 + l).xbuf[4];
            uint32_t* t = (uint32_t*)grow(*dirs[l], sizeof(uint32_t) * (size_t)R * 33 * dstride[l]);
            launch_prescramble(E.d_dv, qc.salt_base + (uint32_t)(l * R), R, dstride[l], t, s0);
        }
        for (size_t q = 0; q < kps.size(); q++) {
            const int l = (int)(q % kBookMaxLevels);
            if (l <= max_L_all) kps[q].dstride = dstride[l];
        }
        if (!kps.empty())
            MCQ_CUDA(cudaMemcpyAsync(grow(*d_kps, sizeof(KParams) * kps.size()), kps.data(), sizeof(KParams) * kps.size(),
                                     cudaMemcpyHostToDevice, s0));
        else
            grow(*d_kps, sizeof(KParams));
        MCQ_CUDA(cudaStreamSynchronize(s0));
        max_specs = (size_t)n * (max_L_all + 1);
        st.assign(n, OptState());
        // chunk records reserved before the timed run (an allocation here can take 0.1 s): the
        // batched rounds' typical need (every slice split kMinChunksPerRep ways), at most 1 GiB,
        // and one slice's worst case per level stream
        const size_t rec = sizeof(double) * kBookNST;
        grow(E.ws(0).xbuf[2], std::min<size_t>(max_specs * (size_t)R * kMinChunksPerRep * rec, (size_t)1 << 30));
        for (int l = 0; l <= max_L_all; l++) grow(E.ws(1 + l).xbuf[2], (size_t)R * kMaxChunksPerRep * rec);
    }

    // The next slices option i needs (run_mlqmc_cuda :1950-2000); steps that need no sample
    // are taken on the host at once.
    void plan(int i) {
        OptState& s = st[i];
        const mcq_book_option& o = opts[i];
        s.n_pending = 0;
        while (!s.done && s.n_pending == 0) {
            if (s.phase == 0) {
                for (int l = 0; l <= 2; l++) add_pending(s, l, ml.pilot_n);
            } else if (s.phase == 2) {
                add_pending(s, s.L, ml.pilot_n);
            } else {
                if (s.iter >= kIterCap) { s.done = true; break; }
                double sum_term = 0.0;
                for (int l = 0; l <= s.L; l++) sum_term += std::sqrt(s.sig2[l] * std::pow((double)M, l));
                for (int l = 0; l <= s.L; l++) {
                    const double Cl = std::pow((double)M, l);
                    long long Nopt = (long long)std::ceil(2.0 / ((double)R * o.eps * o.eps) * std::sqrt(s.sig2[l] / Cl) *
                                                          sum_term);
                    Nopt = std::max(Nopt, 100LL);
                    if (Nopt > s.N[l]) add_pending(s, l, Nopt - s.N[l]);
                }
                if (s.n_pending == 0) end_iteration(i);
            }
        }
    }
    static void add_pending(OptState& s, int l, long long nn) {
        s.pend_level[s.n_pending] = l;
        s.pend_n[s.n_pending++] = nn;
    }

    // Bias test and level growth at the end of an iteration of extras (:1983-1999).
    void end_iteration(int i) {
        OptState& s = st[i];
        const int L = s.L;
        s.iter++;
        double bias = std::abs(s.E[L]) / std::max(M - 1, 1);
        if (L >= 1) bias = std::max(bias, std::abs(s.E[L - 1]) * M / (double)std::max(M * (M - 1), 1));
        if (bias < opts[i].eps / std::sqrt(2.0)) {
            s.done = s.converged = true;
        } else if (L < opts[i].max_L) {
            s.L++;
            s.phase = 2;
        } else if (s.iter >= kIterCap) {
            s.done = true;
        }
    }

    // Merge a slice's {E dY, var of replica means, deltas} into level l (:1927-1944, :1972-1979).
    void absorb(int i, int l, long long nn, const double* r) {
        OptState& s = st[i];
        if (s.N[l] == 0) {
            s.E[l] = r[0];
            s.sig2[l] = r[1] * (double)nn;
            for (int a = 0; a < kMaxBasket; a++) s.Dl[l][a] = r[2 + a];
        } else {
            const double wo = (double)s.N[l], wn = (double)nn;
            s.E[l] = (s.E[l] * wo + r[0] * wn) / (wo + wn);
            s.sig2[l] = (s.sig2[l] * wo + r[1] * wn * wn) / (wo + wn);
            for (int a = 0; a < kMaxBasket; a++) s.Dl[l][a] = (s.Dl[l][a] * wo + r[2 + a] * wn) / (wo + wn);
        }
        s.N[l] += nn;
        s.next_off[l] += nn;
    }

    void step_done(int i) {
        OptState& s = st[i];
        if (s.phase != 1) s.phase = 1;
        else end_iteration(i);
    }

    BookSpec make_spec(int i, int l, long long nn) {
        OptState& s = st[i];
        MCQ_REQUIRE((unsigned long long)(s.next_off[l] + nn) <= 0xFFFFFFFFull, MCQ_ERR_RANGE,
                    "book option " + std::to_string(i) + ": level " + std::to_string(l) +
                        " offset exceeds the 32-bit Sobol limit");
        BookSpec x{};
        x.opt = i;
        x.level = l;
        x.offset = (uint32_t)s.next_off[l];
        x.n_points = (uint32_t)nn;
        // chunk size from the slice alone: at most kChunkNormals normals per lane, split into
        // at least kMinChunksPerRep chunks per replica where the slice has that many groups (a
        // round whose few slices are small still spreads over the GPU), at most kMaxChunksPerRep
        const long long D = (long long)book_width(opts[i]) * nfine(l);
        const uint64_t G = ((uint64_t)x.offset + x.n_points - 1) / 32 + 1 - (x.offset >> 5);
        uint64_t gpc = std::min<uint64_t>((uint64_t)std::max<long long>(1, kChunkNormals / D),
                                          std::max<uint64_t>(1, G / kMinChunksPerRep));
        gpc = std::max<uint64_t>(gpc, (G + kMaxChunksPerRep - 1) / kMaxChunksPerRep);
        x.gpc = (int)gpc;
        x.cpr = (int)((G + gpc - 1) / gpc);
        path_steps += (double)R * (double)nn * (double)(nfine(l) + (l ? nfine(l) / M : 0));
        normals += (double)R * (double)nn * (double)D;
        return x;
    }

    // Order slices by basket width, assign chunk ranges, upload slices and header on s.stream.
    int upload(Slot& s, std::vector<BookSpec>& sp) {
        // by basket width: a class kernel's warps then take chunks of one width at a time, so one
        // specialisation's code is hot in the instruction cache instead of four
        std::stable_sort(sp.begin(), sp.end(), [&](const BookSpec& a, const BookSpec& b) {
            const int ca = book_class_of(opts[a.opt]), cb = book_class_of(opts[b.opt]);
            if (ca != cb) return ca < cb;
            if (ca == kSingleClass)   // one model / payoff's code at a time
                return opts[a.opt].model->kind * 16 + opts[a.opt].payoff->kind <
                       opts[b.opt].model->kind * 16 + opts[b.opt].payoff->kind;
            return opts[a.opt].n_assets < opts[b.opt].n_assets;
        });
        int* h = (int*)s.hspecs.ensure(sizeof(int) * kHdrInts + sizeof(BookSpec) * std::max<size_t>(max_specs, 1));
        std::memset(h, 0, sizeof(int) * kHdrInts);
        BookSpec* hs = reinterpret_cast<BookSpec*>(h + kHdrInts);
        int chunk = 0;
        size_t k = 0;
        for (int c = 0; c < kBookClasses; c++) {
            h[kHdrChunk0 + c] = chunk;
            h[kHdrSlice0 + c] = (int)k;
            for (; k < sp.size() && book_class_of(opts[sp[k].opt]) == c; k++) {
                sp[k].chunk0 = chunk;
                MCQ_REQUIRE((long long)chunk + (long long)R * sp[k].cpr < INT_MAX, MCQ_ERR_RANGE, "book: chunk count overflow");
                chunk += R * sp[k].cpr;
                hs[k] = sp[k];
            }
        }
        h[0] = (int)sp.size();
        h[1] = h[kHdrChunk0 + kBookClasses] = chunk;
        h[kHdrSlice0 + kBookClasses] = (int)sp.size();
        s.specs.ensure(sizeof(BookSpec) * std::max<size_t>(max_specs, 1));
        s.hdr.ensure(sizeof(int) * kHdrInts);
        s.out.ensure(sizeof(double) * kBookOut * std::max<size_t>(max_specs, 1));
        MCQ_CUDA(cudaMemcpyAsync(s.hdr.p, h, sizeof(int) * kHdrInts, cudaMemcpyHostToDevice, s.stream));
        if (!sp.empty())
            MCQ_CUDA(cudaMemcpyAsync(s.specs.p, hs, sizeof(BookSpec) * sp.size(), cudaMemcpyHostToDevice, s.stream));
        return chunk;
    }

    static int grid_of(int cls, int variant) {
        static int per_sm[kBookClasses][kBookVariants] = {{-1, -1}, {-1, -1}, {-1, -1}, {-1, -1}, {-1, -1}};
        if (per_sm[cls][variant] < 0) {
            const void* fn = (const void*)book_fn(cls, variant);
            MCQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)book_smem(cls)));
            int b = 0;
            MCQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kThreads, book_smem(cls)));
            MCQ_REQUIRE(b > 0, MCQ_ERR_INTERNAL, "book kernel does not fit on an SM");
            per_sm[cls][variant] = b;
        }
        return per_sm[cls][variant] * engine().sm_count;
    }

    void launch_book(int cls, int variant, const BookArgs& a, int grid, cudaStream_t st_) {
        void* argv[] = {(void*)&a};
        MCQ_CUDA(cudaLaunchKernel((const void*)book_fn(cls, variant), dim3(grid), dim3(kThreads), argv,
                                 book_smem(cls), st_));
    }
    // a per-slice launch of one class: the tuner's pick, timed while it is still trying variants
    void launch_book_tuned(int cls, const BookArgs& a, int chunks, double normals, cudaStream_t st_) {
        TuneState* trial = nullptr;
        const int v = tune_pick(book_tune_key(cls), kBookVariants, normals, (double)(1 << 26), &trial);
        const int grid = std::max(1, std::min(grid_of(cls, v), (chunks + kWarpsPerBlock - 1) / kWarpsPerBlock));
        if (trial) MCQ_CUDA(cudaEventRecord(trial->ev[v][0], st_));
        launch_book(cls, v, a, grid, st_);
        if (trial) MCQ_CUDA(cudaEventRecord(trial->ev[v][1], st_));
    }
    void launch_fin(const BookArgs& a, int grid, cudaStream_t st_) {
        void* argv[] = {(void*)&a};
        MCQ_CUDA(cudaLaunchKernel((const void*)k_book_fin, dim3(grid), dim3(32 * a.R), argv, 0, st_));
    }

    // ---- batched: one graph per book, replayed once per round
    void run_batched() {
        Engine& E = engine();
        Slot s(E.ws(0));
        constexpr int kSide = kBookClasses - 1;   // class 0 runs on the main stream
        cudaStream_t side[kSide];
        cudaEvent_t fork = nullptr, join[kSide] = {};
        for (int c = 0; c < kSide; c++) side[c] = E.ws(1 + c).stream;
        MCQ_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
        for (auto& e : join) MCQ_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        cudaGraphExec_t exec = nullptr;
        const void* captured_records = nullptr;
        int grid[kBookClasses], var[kBookClasses];
        std::vector<BookSpec> sp;
        auto cleanup = [&]() {
            if (exec) cudaGraphExecDestroy(exec);
            cudaEventDestroy(fork);
            for (auto& e : join) cudaEventDestroy(e);
        };
        try {
            for (;;) {
                sp.clear();
                for (int i = 0; i < n; i++) {
                    plan(i);
                    for (int k = 0; k < st[i].n_pending; k++) sp.push_back(make_spec(i, st[i].pend_level[k], st[i].pend_n[k]));
                }
                if (sp.empty()) break;
                long long chunks = 0;
                for (auto& x : sp) chunks += (long long)R * x.cpr;
                grow(s.records, sizeof(double) * kBookNST * (size_t)std::max<long long>(chunks, 1));
                upload(s, sp);
                bool var_changed = false;
                for (int c = 0; c < kBookClasses; c++) var_changed |= exec && var[c] != book_variant(c);
                // (re)capture when a buffer moved or the tuner settled a class on another variant
                if (!exec || captured_records != s.records.p || var_changed) {
                    if (exec) { MCQ_CUDA(cudaGraphExecDestroy(exec)); exec = nullptr; }
                    for (int c = 0; c < kBookClasses; c++) {
                        var[c] = book_variant(c);
                        grid[c] = grid_of(c, var[c]);
                    }
                    const BookArgs a = args(s);
                    cudaGraph_t g = nullptr;
                    MCQ_CUDA(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
                    MCQ_CUDA(cudaEventRecord(fork, s.stream));
                    for (int c = 0; c < kSide; c++) MCQ_CUDA(cudaStreamWaitEvent(side[c], fork, 0));
                    for (int c = kBookClasses - 1; c >= 1; c--) launch_book(c, var[c], a, grid[c], side[c - 1]);
                    launch_book(0, var[0], a, grid[0], s.stream);
                    for (int c = 0; c < kSide; c++) {
                        MCQ_CUDA(cudaEventRecord(join[c], side[c]));
                        MCQ_CUDA(cudaStreamWaitEvent(s.stream, join[c], 0));
                    }
                    launch_fin(a, E.sm_count * 4, s.stream);
                    MCQ_CUDA(cudaStreamEndCapture(s.stream, &g));
                    const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
                    cudaGraphDestroy(g);
                    MCQ_CUDA(ie);
                    captured_records = s.records.p;
                }
                MCQ_CUDA(cudaGraphLaunch(exec, s.stream));
                double* ho = (double*)s.hout.ensure(sizeof(double) * kBookOut * std::max<size_t>(max_specs, 1));
                MCQ_CUDA(cudaMemcpyAsync(ho, s.out.p, sizeof(double) * kBookOut * sp.size(), cudaMemcpyDeviceToHost,
                                         s.stream));
                MCQ_CUDA(cudaStreamSynchronize(s.stream));
                launches += kBookClasses + 1;
                rounds++;
                for (size_t k = 0; k < sp.size(); k++) absorb(sp[k].opt, sp[k].level, sp[k].n_points, ho + k * kBookOut);
                for (int i = 0; i < n; i++)
                    if (!st[i].done && st[i].n_pending > 0) step_done(i);
            }
        } catch (...) {
            cudaStreamSynchronize(s.stream);
            cleanup();
            throw;
        }
        cleanup();
    }

    // ---- plain: per option, one launch of the option's class kernel per level on its stream
    void run_plain() {
        Engine& E = engine();
        std::vector<Slot> slots;
        slots.reserve(max_L_all + 1);
        for (int l = 0; l <= max_L_all; l++) slots.emplace_back(E.ws(1 + l));
        std::vector<BookSpec> one(1);
        for (int i = 0; i < n; i++) {
            const int cls = book_class_of(opts[i]);
            for (;;) {
                plan(i);
                OptState& s = st[i];
                if (s.done) break;
                int issued_l[kBookMaxLevels];
                long long issued_n[kBookMaxLevels];
                const int np = s.n_pending;
                for (int k = 0; k < np; k++) {
                    const int l = s.pend_level[k];
                    Slot& sl = slots[l];
                    one[0] = make_spec(i, l, s.pend_n[k]);
                    grow(sl.records, sizeof(double) * kBookNST * (size_t)R * one[0].cpr);
                    const int chunks = upload(sl, one);
                    const BookArgs a = args(sl);
                    launch_book_tuned(cls, a, chunks,
                                      (double)R * (double)one[0].n_points * (double)book_width(opts[i]) * (double)nfine(l),
                                      sl.stream);
                    launch_fin(a, 1, sl.stream);
                    double* ho = (double*)sl.hout.ensure(sizeof(double) * kBookOut);
                    MCQ_CUDA(cudaMemcpyAsync(ho, a.out, sizeof(double) * kBookOut, cudaMemcpyDeviceToHost, sl.stream));
                    issued_l[k] = l;
                    issued_n[k] = s.pend_n[k];
                    launches += 2;
                }
                for (int k = 0; k < np; k++) {
                    MCQ_CUDA(cudaStreamSynchronize(slots[issued_l[k]].stream));
                    absorb(i, issued_l[k], issued_n[k], (const double*)slots[issued_l[k]].hout.p);
                }
                rounds++;
                step_done(i);
            }
        }
    }

    void results(mcq_book_result* out) const {
        for (int i = 0; i < n; i++) {
            const OptState& s = st[i];
            mcq_book_result& r = out[i];
            std::memset(&r, 0, sizeof(r));
            double vs = 0.0;
            long long Nt = 0;
            for (int l = 0; l <= s.L; l++) {   // :2010-2016
                r.price += s.E[l];
                if (s.N[l]) vs += s.sig2[l] / ((double)s.N[l] * (double)R);
                Nt += s.N[l] * R;
                if (!opts[i].model)
                    for (int a = 0; a < opts[i].n_assets; a++) r.delta[a] += s.Dl[l][a];
            }
            r.std_error = std::sqrt(vs);
            r.n_samples = Nt;
            r.levels = s.L + 1;
            r.converged = s.converged ? 1 : 0;
        }
    }
};

void book_level_sums(const mcq_book_option& opt, const mcq_mlmc_cfg& ml, const mcq_qmc_cfg& qc, int level,
                     uint32_t offset, long long n_points, double* sums_host) {
    MCQ_REQUIRE(level >= 0 && level <= opt.max_L, MCQ_ERR_INVALID, "book: level beyond the option's max_L");
    MCQ_REQUIRE(n_points >= 1, MCQ_ERR_INVALID, "book: n_points >= 1");
    BookRunner b;
    b.opts = &opt;
    b.n = 1;
    b.ml = ml;
    b.qc = qc;
    b.setup();
    b.st[0].next_off[level] = offset;
    Slot s(engine().ws(0));
    std::vector<BookSpec> one(1, b.make_spec(0, level, n_points));
    grow(s.records, sizeof(double) * kBookNST * (size_t)b.R * one[0].cpr);
    const int chunks = b.upload(s, one);
    const int cls = book_class_of(opt);
    b.launch_book_tuned(cls, b.args(s), chunks, (double)b.R * (double)n_points * (double)book_width(opt) * (double)b.nfine(level),
                        s.stream);
    std::vector<double> rec((size_t)chunks * kBookNST);
    MCQ_CUDA(cudaMemcpyAsync(rec.data(), s.records.p, sizeof(double) * rec.size(), cudaMemcpyDeviceToHost, s.stream));
    MCQ_CUDA(cudaStreamSynchronize(s.stream));
    engine().launches += 1;
    // the summation order of k_book_fin: per lane l the chunks l, l + 32, ..., then the xor butterfly
    const int cpr = one[0].cpr;
    for (int r = 0; r < b.R; r++)
        for (int q = 0; q < kBookNST; q++) {
            double part[32];
            for (int l = 0; l < 32; l++) {
                double v = 0.0;
                for (int j = l; j < cpr; j += 32) v += rec[(size_t)(r * cpr + j) * kBookNST + q];
                part[l] = v;
            }
            for (int off = 16; off > 0; off >>= 1) {
                double nxt[32];
                for (int l = 0; l < 32; l++) nxt[l] = part[l] + part[l ^ off];
                std::memcpy(part, nxt, sizeof(part));
            }
            sums_host[(size_t)r * kBookNST + q] = part[0];
        }
}

void book_price(const mcq_book_option* opts, int n, const mcq_mlmc_cfg& ml, const mcq_qmc_cfg& qc, int mode,
                mcq_book_result* out, mcq_book_stats* stats) {
    MCQ_REQUIRE(out, MCQ_ERR_INVALID, "book: needs an output array");
    MCQ_REQUIRE(mode == MCQ_BOOK_BATCHED || mode == MCQ_BOOK_PLAIN, MCQ_ERR_INVALID, "book: unknown mode");
    const auto t0 = std::chrono::steady_clock::now();
    BookRunner b;
    b.opts = opts;
    b.n = n;
    b.ml = ml;
    b.qc = qc;
    b.setup();
    const auto t1 = std::chrono::steady_clock::now();
    if (mode == MCQ_BOOK_BATCHED) b.run_batched();
    else b.run_plain();
    MCQ_CUDA(cudaDeviceSynchronize());
    MCQ_CUDA(cudaGetLastError());
    const auto t2 = std::chrono::steady_clock::now();
    b.results(out);
    engine().launches += (int)b.launches;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->time_s = std::chrono::duration<double>(t2 - t1).count();
        stats->setup_s = std::chrono::duration<double>(t1 - t0).count();
        stats->path_steps = b.path_steps;
        stats->normals = b.normals;
        stats->rounds = (int)b.rounds;
        stats->launches = (int)b.launches;
    }
}

}  // namespace mcq
