// adjoint.h — the pathwise adjoint pass (k_adjoint.cu).
#pragma once
#include <cstddef>

namespace mcq {

// variant: the checkpoint interval (0: 16 steps, 1: 32, 2: 8; Heston has one)
const void* lookup_adjoint(int model, int payoff, int variant);
size_t adjoint_smem_bytes(int model, int n_steps, int n_nodes, int variant);
int adjoint_variants(int model);

}  // namespace mcq
