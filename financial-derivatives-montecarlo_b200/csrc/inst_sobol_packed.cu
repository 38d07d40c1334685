#include "inst_common.cuh"
namespace mcq {
// Raw-ordered passes of paths with at most 16 normals (NOISE_PACKED), plain and coupled.
const void* lookup_sobol_packed(int model, int pay, bool coupled) {
    if (coupled) {
        switch (model) {
            case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_PACKED, MOD_GBM, true>(pay);
            case MOD_HESTON: return pick_payoff<GEN_SOBOL, NOISE_PACKED, MOD_HESTON, true>(pay);
            case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_PACKED, MOD_DUPIRE, true>(pay);
            default: return nullptr;
        }
    }
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_PACKED, MOD_GBM, false>(pay);
        case MOD_HESTON: return pick_payoff<GEN_SOBOL, NOISE_PACKED, MOD_HESTON, false>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_PACKED, MOD_DUPIRE, false>(pay);
        case MOD_LVGRID: return pick_payoff<GEN_SOBOL, NOISE_PACKED, MOD_LVGRID, false>(pay);
        default: return nullptr;
    }
}
}  // namespace mcq
