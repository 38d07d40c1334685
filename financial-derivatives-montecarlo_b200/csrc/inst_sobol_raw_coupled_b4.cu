// Register-budget variant (4 resident CTAs per SM, 64 registers) of the coupled fine / coarse
// Sobol raw-noise pass family (the MLMC / MLQMC levels); chosen per family by the engine's
// autotuner (engine.cpp).
#include "inst_common.cuh"
namespace mcq {
const void* lookup_sobol_raw_coupled_b4(int model, int pay) {
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_GBM, true, 4>(pay);
        case MOD_HESTON: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_HESTON, true, 4>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_DUPIRE, true, 4>(pay);
        default: return nullptr;
    }
}
}  // namespace mcq
