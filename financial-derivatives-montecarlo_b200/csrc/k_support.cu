// k_support.cu — small kernels around the fused pass: per-replica direction-word scrambling,
// the deterministic cross-item reduction, and the Sobol stream export used by parity tests.
#include <cuda_runtime.h>
#include <cstdint>
#include "path_kernels.cuh"
#include "support.h"

namespace mcq {

// Pre-scrambled direction words for salts salt0 .. salt0+R-1 and dims 0..D-1:
// out[r][k][d] = hh_linear(v[d][k], splitmix32(salt) ^ d) for k < 32, and the digital shift
// splitmix32(base ^ 0xA5A5A5A5) at k = 32 (methods_cuda.cu:786-795, :819).
__global__ void k_prescramble(const uint32_t* __restrict__ dv, uint32_t salt0, int R, int D,
                              uint32_t* __restrict__ out) {
    const long long total = (long long)R * 33 * D;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / (33LL * D));
        const int rem = (int)(idx - (long long)r * 33 * D);
        const int k = rem / D, d = rem - k * D;
        const uint32_t base = splitmix32(salt0 + (uint32_t)r) ^ (uint32_t)d;
        out[idx] = (k < 32) ? hh_linear(__ldg(dv + (size_t)d * 32 + k), base)
                            : splitmix32(base ^ 0xA5A5A5A5u);
    }
}

// out[r][s] = sum over j of partials[(r * ipr + j) * nstat + s]; fixed summation order.
__global__ void k_finalize(const double* __restrict__ partials, int ipr, int nstat,
                           double* __restrict__ out) {
    __shared__ double red[256];
    const int r = blockIdx.x, t = threadIdx.x;
    for (int s = 0; s < nstat; s++) {
        double v = 0.0;
        for (int j = t; j < ipr; j += 256) v += partials[((size_t)r * ipr + j) * nstat + s];
        red[t] = v;
        __syncthreads();
        for (int o = 128; o > 0; o >>= 1) {
            if (t < o) red[t] += red[t + o];
            __syncthreads();
        }
        if (t == 0) out[(size_t)r * nstat + s] = red[0];
        __syncthreads();
    }
}

// Scrambled integers / normals of one replica by the direct gray-code form:
// out[d * n + i] for dim dim0 + d and point offset + i.
__global__ void k_sobol_export(const uint32_t* __restrict__ tab, int D, int dim0, int nd,
                               uint32_t offset, long long n, float u_cap, int as_normal,
                               void* out) {
    const long long total = (long long)nd * n;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int d = (int)(idx / n);
        const long long i = idx - (long long)d * n;
        const int dim = dim0 + d;
        const uint32_t pt = offset + (uint32_t)i;
        uint32_t g = pt ^ (pt >> 1);
        uint32_t x = __ldg(tab + 32 * D + dim);
        while (g) {
            const int k = __ffs(g) - 1;
            x ^= __ldg(tab + k * D + dim);
            g &= g - 1;
        }
        if (as_normal) static_cast<float*>(out)[idx] = sobol_normal(x, u_cap);
        else static_cast<uint32_t*>(out)[idx] = x;
    }
}

void launch_prescramble(const uint32_t* dv, uint32_t salt0, int R, int D, uint32_t* out,
                        cudaStream_t s) {
    const long long total = (long long)R * 33 * D;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_prescramble<<<blocks, 256, 0, s>>>(dv, salt0, R, D, out);
}

void launch_finalize(const double* partials, int R, int ipr, int nstat, double* out,
                     cudaStream_t s) {
    k_finalize<<<R, 256, 0, s>>>(partials, ipr, nstat, out);
}

void launch_sobol_export(const uint32_t* tab, int D, int dim0, int nd, uint32_t offset,
                         long long n, float u_cap, int as_normal, void* out, cudaStream_t s) {
    const long long total = (long long)nd * n;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    k_sobol_export<<<blocks, 256, 0, s>>>(tab, D, dim0, nd, offset, n, u_cap, as_normal, out);
}

// Failure-path probe of the bounded mbarrier wait that the assisted passes (and, with the same
// limit logic, the tensor-core PCA pass) use: one warp waits on a barrier that nothing arrives on,
// gives up after `polls` polls and records MCQ_ERR_TIMEOUT in the status word, which the host's
// check turns into the API error.  No fault, no hang: the wait always returns.
__global__ void k_wait_probe(int* err, uint32_t polls) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(asst_addr(&bar)), "r"(1));
    __syncthreads();
    const bool ok = asst_wait(&bar, 0u, polls);
    if (!__all_sync(0xffffffffu, ok) && threadIdx.x == 0) atomicExch(err, MCQ_ERR_TIMEOUT_CODE);
}

void launch_wait_probe(int* err, uint32_t polls, cudaStream_t s) {
    k_wait_probe<<<1, 32, 0, s>>>(err, polls);
}

// Time rows of the grid local-vol model for steps 0 .. n - 1 of a pass (lv_time_row).
__global__ void k_lv_rows(const __grid_constant__ KParams p, float2* rows, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        rows[k] = lv_time_row(p, k);
}

void launch_lv_rows(const KParams& p, float2* rows, int n, cudaStream_t s) {
    k_lv_rows<<<(n + 255) / 256, 256, 0, s>>>(p, rows, n);
}

}  // namespace mcq
