// pca_large.cu — PCA ordering for step counts the tensor-core pass cannot hold.
//
// k_pca keeps the whole N x N fp16 PCA factor in shared memory, which bounds it to N <= 256
// (N in {64, 128, 256}; N <= 32 runs inside k_pass).  Every other N (the reference's examples
// size their QMC PCA runs up to 2048 steps, and its MLQMC PCA levels up to 512) runs here in
// three steps per batch of points of one replica, the reference's own structure
// (methods_cuda.cu:1150-1166, :1228-1229) without its HBM round trips for the other stages:
//   1. k_pca_normals: the scrambled-Sobol normals of the batch, rounded to fp16 (as the
//      reference's cast kernel), written as Z[k][row] (column-major, rows = points);
//   2. one plain library GEMM, dW = Z M^T in fp32 (fp16 inputs, FP32 accumulation), as the
//      reference's cublasGemmEx;
//   3. the fused pass in NOISE_DW mode: each lane reads its path's increments in time order and
//      runs the model, payoff and reductions; the batch's per-replica sums are added into the
//      caller's output.
// Batches hold at most kBatchFloats / N points so that Z and dW stay a few hundred MB.
#include <cublas_v2.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "dispatch.h"
#include "engine.h"
#include "path_kernels.cuh"
#include "pca.h"
#include "support.h"

namespace mcq {

namespace {
constexpr long long kBatchFloats = 1LL << 27;   // Z: 256 MB fp16, dW: 512 MB fp32 at most

// One warp per (32-point group, 32-dimension tile): the tile's normals through the transpose
// buffer, then lane l writes point 32h + l of each of the 32 dimensions (consecutive rows per
// dimension: coalesced).
__global__ void __launch_bounds__(kThreads) k_pca_normals(const uint32_t* __restrict__ dr, int N, uint64_t g0,
                                                         uint64_t G, uint64_t offset, uint64_t n_points,
                                                         float u_cap, __half* __restrict__ Z, int ldz) {
    __shared__ float tile[kWarpsPerBlock][1024];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    float* buf = tile[wib];
    const int ntiles = (N + 31) >> 5;
    const uint64_t tasks = G * (uint64_t)ntiles;
    for (uint64_t t = (uint64_t)blockIdx.x * kWarpsPerBlock + wib; t < tasks;
         t += (uint64_t)gridDim.x * kWarpsPerBlock) {
        const uint64_t h = g0 + t / (uint64_t)ntiles;
        const int d0 = (int)(t % (uint64_t)ntiles) * 32;
        sobol_tile(dr, N, d0 + lane, d0 + lane < N, h, u_cap, buf, lane);
        __syncwarp();
        float z[32];
        read_row(buf, lane, z);
        __syncwarp();
        const uint64_t n = h * 32 + (uint64_t)lane;
        if (n >= offset && n < offset + n_points) {
            const size_t row = (size_t)(n - offset);
#pragma unroll
            for (int c = 0; c < 32; c++)
                if (d0 + c < N) Z[(size_t)(d0 + c) * (size_t)ldz + row] = __float2half_rn(z[c]);
        }
    }
}

__global__ void k_add_sums(double* __restrict__ dst, const double* __restrict__ src, int n) {
    const int i = threadIdx.x;
    if (i < n) dst[i] += src[i];
}

void cublas_check(cublasStatus_t s, const char* what) {
    MCQ_REQUIRE(s == CUBLAS_STATUS_SUCCESS, MCQ_ERR_CUDA, std::string("cuBLAS ") + what + " failed (status " +
                                                              std::to_string((int)s) + ")");
}
}  // namespace

Workspace::Blas::~Blas() {
    if (h) cublasDestroy(static_cast<cublasHandle_t>(h));
}

void pca_large_pass_async(Workspace& ws, const PassArgs& a, KParams& k, double* d_out) {
    Engine& E = engine();
    const int N = k.D;
    const int R = a.R;
    const int nst = k.nstat;
    const void* fn = lookup_dw(k.model, a.p->kind, a.est == EST_COUPLED);
    MCQ_REQUIRE(fn != nullptr, MCQ_ERR_UNSUPPORTED, "no PCA pass for this model / payoff");
    if (!ws.blas.h) {
        cublasHandle_t h = nullptr;
        cublas_check(cublasCreate(&h), "create");
        ws.blas.h = h;
    }
    cublasHandle_t blas = static_cast<cublasHandle_t>(ws.blas.h);
    cublas_check(cublasSetStream(blas, ws.stream), "set stream");

    if (!(ws.dirs_salt0 == a.salt0 && ws.dirs_R == R && ws.dirs_D == N)) {
        uint32_t* d = (uint32_t*)ws.dirs.ensure(sizeof(uint32_t) * (size_t)R * 33 * N);
        launch_prescramble(E.d_dv, a.salt0, R, N, d, ws.stream);
        E.launches++;
        ws.dirs_salt0 = a.salt0;
        ws.dirs_R = R;
        ws.dirs_D = N;
    }
    const uint32_t* dirs = (const uint32_t*)ws.dirs.p;
    const uint64_t pb = std::max<uint64_t>(32, (uint64_t)(kBatchFloats / N) / 32 * 32);
    const uint64_t pfirst = std::min<uint64_t>(pb, (a.n_points + 31) / 32 * 32);
    __half* Z = (__half*)ws.pca_z.ensure(sizeof(__half) * (size_t)pfirst * N);
    float* dW = (float*)ws.pca_dw.ensure(sizeof(float) * (size_t)pfirst * N);
    double* tmp = (double*)ws.pca_tmp.ensure(sizeof(double) * nst);
    MCQ_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * (size_t)R * nst, ws.stream));
    const size_t csmem = (size_t)kWarpsPerBlock * 1024 * sizeof(float);
    KernelInfo& ki = kernel_info(fn, csmem);
    const float one = 1.0f, zero = 0.0f;
    for (int r = 0; r < R; r++) {
        const uint32_t* dr = dirs + (size_t)r * 33 * N;
        for (uint64_t o = a.offset; o < a.offset + a.n_points; o += pb) {
            const uint64_t nb = std::min<uint64_t>(pb, a.offset + a.n_points - o);
            const int ld = (int)((nb + 31) / 32 * 32);
            const uint64_t g0 = o >> 5;
            const uint64_t G = ((o + nb - 1) >> 5) - g0 + 1;
            const uint64_t tasks = G * (uint64_t)((N + 31) >> 5);
            const long long gblocks = std::min<long long>((long long)((tasks + kWarpsPerBlock - 1) / kWarpsPerBlock),
                                                          (long long)E.sm_count * 8);
            k_pca_normals<<<(unsigned)std::max<long long>(gblocks, 1), kThreads, 0, ws.stream>>>(
                dr, N, g0, G, o, nb, k.u_cap, Z, ld);
            MCQ_CUDA(cudaGetLastError());
            // dW (ld x N, column-major) = Z (ld x N) * B, B(k, i) = M[i][k] = table[i * N + k]
            cublas_check(cublasGemmEx(blas, CUBLAS_OP_N, CUBLAS_OP_N, ld, N, N, &one, Z, CUDA_R_16F, ld, a.pca->table.p,
                                      CUDA_R_16F, N, &zero, dW, CUDA_R_32F, ld, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT),
                         "GemmEx");
            KParams kc = k;
            kc.noise = NOISE_DW;
            kc.R = 1;
            kc.offset = o;
            kc.n_points = nb;
            kc.g0 = g0;
            kc.G = G;
            uint64_t gpi = (G + kTargetItems - 1) / kTargetItems;
            if (gpi < 1) gpi = 1;
            const uint64_t ipr = (G + gpi - 1) / gpi;
            kc.gpi = (int)gpi;
            kc.items_per_rep = (int)ipr;
            kc.n_items = (int)ipr;
            kc.dw_in = dW;
            kc.dw_stride = ld;
            kc.partials = (double*)ws.partials.ensure(sizeof(double) * (size_t)ipr * nst);
            long long blocks = std::min<long long>(((long long)ipr + kWarpsPerBlock - 1) / kWarpsPerBlock,
                                                   (long long)ki.blocks_per_sm * E.sm_count);
            void* args[] = {&kc};
            MCQ_CUDA(cudaLaunchKernel(fn, dim3((unsigned)std::max<long long>(blocks, 1)), dim3(kThreads), args, csmem,
                                      ws.stream));
            launch_finalize(kc.partials, 1, (int)ipr, nst, tmp, ws.stream);
            k_add_sums<<<1, 32, 0, ws.stream>>>(d_out + (size_t)r * nst, tmp, nst);
            MCQ_CUDA(cudaGetLastError());
            E.launches += 4;
        }
    }
}

}  // namespace mcq
