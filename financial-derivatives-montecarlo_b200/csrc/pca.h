// pca.h — the tensor-core PCA pass (k_pca.cu): kernel lookup and launch geometry.
#pragma once
#include <cstddef>

#include "kparams.h"

namespace mcq {

const void* lookup_pca(int model, int payoff, bool coupled, bool dump);   // nullptr: unsupported
size_t pca_smem_bytes(int N);   // dynamic shared memory of a launch
int pca_threads();      // block size
int pca_warps();        // per-warp records per work item
int pca_tile_paths();   // paths per tile

}  // namespace mcq
