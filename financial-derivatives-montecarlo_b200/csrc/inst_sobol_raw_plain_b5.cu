// Register-budget variant (5 resident CTAs per SM, 48 registers) of the single-level Sobol
// raw-noise pass family; chosen per family by the engine's autotuner (engine.cpp).
#include "inst_common.cuh"
namespace mcq {
const void* lookup_sobol_raw_plain_b5(int model, int pay) {
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_GBM, false, 5>(pay);
        case MOD_HESTON: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_HESTON, false, 5>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_DUPIRE, false, 5>(pay);
        case MOD_LVGRID: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_LVGRID, false, 5>(pay);
        default: return nullptr;
    }
}
}  // namespace mcq
