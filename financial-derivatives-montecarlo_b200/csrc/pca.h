// pca.h — the tensor-core PCA pass (k_pca.cu): kernel lookup and launch geometry.
#pragma once
#include <cstddef>

namespace mcq {

// Status written to KParams::err when a bounded device wait gives up (MCQ_ERR_TIMEOUT).
constexpr int MCQ_ERR_TIMEOUT_CODE = 7;

const void* lookup_pca(int model, int payoff, bool coupled, bool dump);
size_t pca_smem_bytes(int N);
int pca_threads();
int pca_warps();

}  // namespace mcq
