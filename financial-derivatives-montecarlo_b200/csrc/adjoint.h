// adjoint.h — the pathwise adjoint pass (k_adjoint.cu).
#pragma once
#include <cstddef>

namespace mcq {

const void* lookup_adjoint(int model, int payoff);
size_t adjoint_smem_bytes(int model, int n_steps, int n_nodes);

}  // namespace mcq
