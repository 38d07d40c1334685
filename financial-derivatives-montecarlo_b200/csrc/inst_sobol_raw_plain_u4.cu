// Code-shape variant of the single-level Sobol raw-noise pass family: 4 resident CTAs per SM
// (64 registers) with the tile generator's four blocks of eight points unrolled (fewer loop
// instructions, more inlined inverse-normal code); chosen per family by the engine's autotuner
// (engine.cpp).  The same normals and sums as the other variants.
#include "inst_common.cuh"
namespace mcq {
const void* lookup_sobol_raw_plain_u4(int model, int pay) {
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_GBM, false, 4, 4>(pay);
        case MOD_HESTON: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_HESTON, false, 4, 4>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_DUPIRE, false, 4, 4>(pay);
        case MOD_LVGRID: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_LVGRID, false, 4, 4>(pay);
        default: return nullptr;
    }
}
}  // namespace mcq
