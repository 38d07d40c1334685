// Register-budget variant (3 resident CTAs per SM, 85 registers) of the single-level Sobol
// Brownian-bridge pass family; chosen per family by the engine's autotuner (engine.cpp).
#include "inst_common.cuh"
namespace mcq {
const void* lookup_sobol_bb_b3(int model, int pay) {
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_BB, MOD_GBM, false, 3>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_BB, MOD_DUPIRE, false, 3>(pay);
        case MOD_LVGRID: return pick_payoff<GEN_SOBOL, NOISE_BB, MOD_LVGRID, false, 3>(pay);
        default: return nullptr;
    }
}
}  // namespace mcq
