// Code-shape variant of the coupled fine / coarse Sobol raw-noise pass family (the MLMC / MLQMC
// levels): 4 resident CTAs per SM (64 registers) with the tile generator's four blocks of eight
// points unrolled; chosen per family by the engine's autotuner (engine.cpp).  The same normals
// and sums as the other variants.
#include "inst_common.cuh"
namespace mcq {
const void* lookup_sobol_raw_coupled_u4(int model, int pay) {
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_GBM, true, 4, 4>(pay);
        case MOD_HESTON: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_HESTON, true, 4, 4>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_RAW, MOD_DUPIRE, true, 4, 4>(pay);
        default: return nullptr;
    }
}
}  // namespace mcq
