// k_pca.cu — the PCA-ordered RQMC pass on the 5th-generation tensor cores (sm_100a).
//
// The reference applies PCA as three HBM passes: cast the normals to fp16, one cuBLAS GEMM
// dW = Z M^T over the whole [D x N] array, then the path kernel (methods_cuda.cu:1150-1166,
// :1228-1229, :720-724).  Here one persistent, warp-specialised kernel does it per tile of 128
// paths (one M = 128 MMA), with the PCA factor M (fp16, N x N) resident in shared memory:
//   * 24 generator warps make the tile's scrambled-Sobol normals, 64 dimensions (one K-block) at
//     a time: a K-block is eight work units of 32 paths x 32 dimensions, one per warp of a group
//     of eight, and the three groups take every third K-block.  They store the normals as fp16
//     (round to nearest, as __float2half in the reference) straight into a 128-byte-swizzled
//     K-major stage of a four-stage ring and arrive on the stage's `full` barrier;
//   * one issuer thread waits for a stage, issues tcgen05.mma kind::f16 (fp16 x fp16 -> fp32)
//     against M, and releases the stage with tcgen05.commit on its `empty` barrier; after a
//     tile's last K-block it commits the tile's accumulator;
//   * the accumulator is double-buffered in tensor memory (2 x N columns): four drain warps (one
//     per TMEM lane quarter) read their 32 paths' lanes with tcgen05.ld (32 time steps at a
//     time), feed the increments to the path consumer and release the accumulator, so that a
//     tile's drain overlaps the next tile's generation and MMA.
// The normal generation bounds the kernel (the path consumer is a small fraction of the
// instructions), so most warps generate: 4 drain + 24 generator warps + 1 issuer warp, 928
// threads at up to 64 registers; 16 generators with 8 drain warps ran 19 % slower.
// Every mbarrier wait is bounded: after the limit the CTA records MCQ_ERR_TIMEOUT in p.err, the
// issuer waits (bounded) for its MMAs in flight, and the CTA frees its TMEM and returns.
//
// Supported sizes: N = D in {64, 128, 256} (K-blocks of 64, MMA N <= 256).
#include <cuda_fp16.h>

#include "path_kernels.cuh"
#include "pca.h"

namespace mcq {

constexpr int kPcaDrainWarps = 4;            // warps 0-3: one per TMEM lane quarter
constexpr int kPcaGenWarps = 24;             // warps 4-27: three groups of eight
constexpr int kPcaGroups = kPcaGenWarps / 8;
constexpr int kPcaIssuerWarp = kPcaDrainWarps + kPcaGenWarps;
constexpr int kPcaThreads = (kPcaIssuerWarp + 1) * 32;
constexpr int kPcaRows = 128;                // paths per tile: one M = 128 MMA
constexpr int kPcaStages = 4;                // ring of K-block stages
constexpr int kAStageBytes = kPcaRows * 128; // 128 rows x 64 fp16
constexpr uint32_t kWaitLimit = 1u << 26;    // polls of an mbarrier before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
    return (uint32_t)__cvta_generic_to_shared(ptr);
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t addr) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
}

// Bounded wait for completion of the phase with parity `parity`; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; i++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor, K-major operand in the 128-byte swizzle: 8-row atoms of
// 128 B (1 KiB, the stride between atoms), start address in 16-byte units, descriptor
// version 1 in bits 46-47, layout type SWIZZLE_128B (2) in bits 61-63.  The leading offset is
// not used by this layout (one MMA's K = 16 fp16 = 32 B stays inside the atom).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                        uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar_addr) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            mbar_addr)
        : "memory");
}

// 32 consecutive fp32 columns of this warp's 32 TMEM lanes (one row per thread).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
        "%28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Normals of points 32h..32h+31 for dimension `dim`, stored as fp16 at element e of the
// 64-wide K-block of rows row0..row0+31 in the swizzled tile `A` (row r at r*128 bytes, 16-byte
// chunk c at position c ^ (r & 7)).
__device__ __forceinline__ void sobol_tile_to_A(const uint32_t* __restrict__ dr, int D, int dim,
                                                uint64_t h, float u_cap, unsigned char* A,
                                                int row0, int e) {
    const uint32_t* col = dr + dim;
    const uint32_t L0 = __ldg(col), L1 = __ldg(col + D), L2 = __ldg(col + 2 * D),
                   L3 = __ldg(col + 3 * D), L4 = __ldg(col + 4 * D);
    uint32_t x = __ldg(col + 32 * D);
    if (h & 1) x ^= L4;
    uint32_t g = (uint32_t)(h ^ (h >> 1));
    while (g) {
        const int k = __ffs(g) - 1;
        x ^= __ldg(col + (5 + k) * D);
        g &= g - 1;
    }
    unsigned char* base = A + (e & 7) * 2;
    const int chunk = e >> 3;
    // four blocks of eight points (the gray-code steps as in sobol_tile), unrolled
#pragma unroll
    for (int b = 0; b < 4; b++) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int r = row0 + 8 * b + i;
            *reinterpret_cast<__half*>(base + r * 128 + ((chunk ^ (r & 7)) << 4)) =
                __float2half_rn(sobol_normal(x, u_cap));
            if (i < 7) {
                x ^= gray_word8(i, L0, L1, L2);
            } else if (b < 3) {
                x ^= (b == 1) ? L4 : L3;
            }
        }
    }
}

template <class C>
__global__ void __launch_bounds__(kPcaThreads, 1) k_pca(const __grid_constant__ KParams p) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const uint32_t raw_addr = smem_u32(smem_raw);
    unsigned char* sm = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
    const int N = p.D;
    const int nkb = N >> 6;
    unsigned char* sB = sm;
    unsigned char* sA = sm + N * N * 2;
    uint64_t* full = reinterpret_cast<uint64_t*>(sA + kPcaStages * kAStageBytes);  // stage written
    uint64_t* empty = full + kPcaStages;       // stage read by its MMAs
    uint64_t* accfull = empty + kPcaStages;    // accumulator a holds a finished tile
    uint64_t* accempty = accfull + 2;          // accumulator a drained
    uint64_t* done = accempty + 2;             // every MMA issued has completed
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* s_fail = reinterpret_cast<volatile int*>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ncols = (uint32_t)(2 * N);   // two accumulators of N fp32 columns

    // the PCA factor, row i = output step, K contiguous: 16-byte chunks into the swizzled layout
    {
        const uint4* Bg = reinterpret_cast<const uint4*>(p.pca);
        const int cpr = N >> 3;
        for (int idx = tid; idx < N * cpr; idx += kPcaThreads) {
            const int i = idx / cpr, c16 = idx - i * cpr;
            const int kb = c16 >> 3, c = c16 & 7;
            *reinterpret_cast<uint4*>(sB + kb * (N * 128) + i * 128 + ((c ^ (i & 7)) << 4)) = __ldg(Bg + idx);
        }
    }
    if (tid == 0) {
        for (int s = 0; s < kPcaStages; s++) {
            mbar_init(smem_u32(&full[s]), 8 * 32);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(smem_u32(&accfull[a]), 1);
            mbar_init(smem_u32(&accempty[a]), 4 * 32);
        }
        mbar_init(smem_u32(done), 1);
        *s_fail = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tslot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;

    // Every role walks the same sequence: items blockIdx.x, + gridDim.x, ...; tiles [t_beg, t_end)
    // of each item; q counts the CTA's tiles, K-block kb of tile q is the CTA's K-block q nkb + kb.
    const int tiles_per_rep = (int)((p.G + 3) >> 2);
    const int n_items = p.n_items;
    if (warp < kPcaDrainWarps) {
        // ---- drain warps: every tile, tile q from accumulator q mod 2
        const int quarter = warp;
        const uint32_t tlane = tbase + ((uint32_t)(32 * quarter) << 16);
        int q = 0;
        bool stop = false;
        for (int item = blockIdx.x; item < n_items && !stop; item += gridDim.x) {
            const int r = item / p.items_per_rep;
            const int j = item - r * p.items_per_rep;
            const int t_beg = j * p.gpi;
            const int t_end = min(t_beg + p.gpi, tiles_per_rep);
            Acc<C::NST> acc;
            acc.zero();
            for (int t = t_beg; t < t_end; t++, q++) {
                const int a = q & 1;
                const uint32_t trow = tlane + (uint32_t)(a * N);
                const bool ok = mbar_wait(smem_u32(&accfull[a]), (uint32_t)(q >> 1) & 1u);
                if (!__all_sync(0xffffffffu, ok && !*s_fail)) { *s_fail = 1; stop = true; break; }
                tc_fence_after();
                const uint64_t n = (p.g0 + (uint64_t)t * 4 + (uint64_t)quarter) * 32 + (uint64_t)lane;
                C cons;
                cons.init(p);
                if constexpr (std::is_same<C, DumpC>::value) cons.bind(p, r, n);
                else cons.bind(r, n);
                for (int c0 = 0; c0 < N; c0 += 32) {
                    float v[32];
                    tmem_ld32(trow + (uint32_t)c0, v);
#pragma unroll
                    for (int i = 0; i < 32; i++) cons.step_dw(p, v[i], 0.f);
                    cons.flush();
                }
                tc_fence_before();   // TMEM reads done before the accumulator is released
                mbar_arrive(smem_u32(&accempty[a]));
                float y[C::NST];
                cons.finish(p, y);
                if (n >= p.offset && n < p.offset + p.n_points) acc.add(y);
            }
            if (!stop) acc.flush(p.partials + ((size_t)item * kPcaDrainWarps + warp) * C::NST, lane);
        }
    } else if (warp < kPcaIssuerWarp) {
        // ---- generator warps: group grp (eight warps) makes the K-blocks jj with jj mod (groups) =
        //      grp; warp gi makes unit (row group rg, dimension half hf) of each: rows 32 rg ..
        //      32 rg + 31, dimensions 32 hf .. 32 hf + 31 of the K-block
        const int gi = warp - kPcaDrainWarps;
        const int rg = gi & 3, hf = (gi >> 2) & 1, grp = gi >> 3;
        int q = 0;
        bool stop = false;
        for (int item = blockIdx.x; item < n_items && !stop; item += gridDim.x) {
            const int r = item / p.items_per_rep;
            const int j = item - r * p.items_per_rep;
            const int t_beg = j * p.gpi;
            const int t_end = min(t_beg + p.gpi, tiles_per_rep);
            const uint32_t* dr = p.dirs + (size_t)r * 33 * (size_t)N;
            for (int t = t_beg; t < t_end && !stop; t++, q++) {
                const uint64_t h = p.g0 + (uint64_t)t * 4 + (uint64_t)rg;
                for (int kb = 0; kb < nkb; kb++) {
                    const int jj = q * nkb + kb;
                    if (jj % kPcaGroups != grp) continue;
                    const int s = jj % kPcaStages, u = jj / kPcaStages;
                    if (u > 0) {   // the MMAs of this stage's previous K-block have read it
                        const bool ok = mbar_wait(smem_u32(&empty[s]), (uint32_t)(u - 1) & 1u);
                        if (!__all_sync(0xffffffffu, ok && !*s_fail)) { *s_fail = 1; stop = true; break; }
                    }
                    sobol_tile_to_A(dr, N, kb * 64 + 32 * hf + lane, h, p.u_cap, sA + s * kAStageBytes, 32 * rg,
                                    32 * hf + lane);
                    fence_proxy_async();   // generic-proxy stores visible to the tensor core's reads
                    mbar_arrive(smem_u32(&full[s]));
                }
            }
        }
    } else if (lane == 0) {
        // ---- the issuer thread
        const uint32_t idesc = (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kPcaRows >> 4) << 24);
        const uint32_t sB_addr = smem_u32(sB), sA_addr = smem_u32(sA);
        int q = 0;
        bool stop = false;
        for (int item = blockIdx.x; item < n_items && !stop; item += gridDim.x) {
            const int j = item - (item / p.items_per_rep) * p.items_per_rep;
            const int t_beg = j * p.gpi;
            const int t_end = min(t_beg + p.gpi, tiles_per_rep);
            for (int t = t_beg; t < t_end && !stop; t++, q++) {
                const int a = q & 1;
                if (q >= 2 && (!mbar_wait(smem_u32(&accempty[a]), (uint32_t)((q >> 1) - 1) & 1u) || *s_fail)) {
                    *s_fail = 1;
                    stop = true;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tbase + (uint32_t)(a * N);
                for (int kb = 0; kb < nkb; kb++) {
                    const int jj = q * nkb + kb;
                    const int s = jj % kPcaStages, u = jj / kPcaStages;
                    if (!mbar_wait(smem_u32(&full[s]), (uint32_t)u & 1u) || *s_fail) {
                        *s_fail = 1;
                        stop = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = sA_addr + s * kAStageBytes, b0 = sB_addr + kb * (N * 128);
#pragma unroll
                    for (int ks = 0; ks < 4; ks++)
                        mma_f16(d, sw128_desc(a0 + ks * 32), sw128_desc(b0 + ks * 32), idesc, (kb | ks) != 0 ? 1u : 0u);
                    mma_commit(smem_u32(&empty[s]));
                }
                if (!stop) mma_commit(smem_u32(&accfull[a]));
            }
        }
        // teardown: the commit tracks every MMA issued so far
        mma_commit(smem_u32(done));
        if (!mbar_wait(smem_u32(done), 0u)) *s_fail = 1;
    }
    __syncwarp();   // the issuer warp reconverges
    tc_fence_before();
    __syncthreads();
    if (tid == 0 && *s_fail) atomicExch(p.err, MCQ_ERR_TIMEOUT_CODE);
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(ncols));
    }
}

template <int MOD, bool CPL>
static const void* pca_payoff(int pay) {
    switch (pay) {
        case PAY_EUR:
        case PAY_BASKET: return (const void*)&k_pca<PathC<MOD, PAY_EUR, CPL>>;
        case PAY_ASIAN: return (const void*)&k_pca<PathC<MOD, PAY_ASIAN, CPL>>;
        case PAY_GEOM: return (const void*)&k_pca<PathC<MOD, PAY_GEOM, CPL>>;
        case PAY_LOOKBACK: return (const void*)&k_pca<PathC<MOD, PAY_LOOKBACK, CPL>>;
        case PAY_UPOUT: return (const void*)&k_pca<PathC<MOD, PAY_UPOUT, CPL>>;
        case PAY_DOWNOUT: return (const void*)&k_pca<PathC<MOD, PAY_DOWNOUT, CPL>>;
        default: return nullptr;
    }
}

const void* lookup_pca(int model, int payoff, bool coupled, bool dump) {
    if (dump) return (const void*)&k_pca<DumpC>;
    if (coupled) {
        switch (model) {
            case MOD_GBM: return pca_payoff<MOD_GBM, true>(payoff);
            case MOD_DUPIRE: return pca_payoff<MOD_DUPIRE, true>(payoff);
            default: return nullptr;
        }
    }
    switch (model) {
        case MOD_GBM: return pca_payoff<MOD_GBM, false>(payoff);
        case MOD_DUPIRE: return pca_payoff<MOD_DUPIRE, false>(payoff);
        case MOD_LVGRID: return pca_payoff<MOD_LVGRID, false>(payoff);
        default: return nullptr;
    }
}

size_t pca_smem_bytes(int N) { return (size_t)N * N * 2 + (size_t)kPcaStages * kAStageBytes + 256 + 1024; }
int pca_threads() { return kPcaThreads; }
int pca_warps() { return kPcaDrainWarps; }
int pca_tile_paths() { return kPcaRows; }

}  // namespace mcq
