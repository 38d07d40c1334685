// support.h — host-side launchers for the support kernels in k_support.cu.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace mcq {

void launch_prescramble(const uint32_t* dv, uint32_t salt0, int R, int D, uint32_t* out,
                        cudaStream_t s);
void launch_finalize(const double* partials, int R, int ipr, int nstat, double* out,
                     cudaStream_t s);
// one warp waits `polls` times on an mbarrier nothing arrives on, then records MCQ_ERR_TIMEOUT
void launch_wait_probe(int* err, uint32_t polls, cudaStream_t s);
struct KParams;
// the grid local-vol model's time rows of steps 0 .. n - 1 (lv_time_row) into rows[n]
void launch_lv_rows(const KParams& p, float2* rows, int n, cudaStream_t s);
void launch_sobol_export(const uint32_t* tab, int D, int dim0, int nd, uint32_t offset,
                         long long n, float u_cap, int as_normal, void* out, cudaStream_t s);

}  // namespace mcq
