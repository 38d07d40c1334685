#include "inst_common.cuh"
namespace mcq {
// Brownian-bridge passes with uniform window weights (NOISE_BB_UNI): plain at 3 and 4 resident CTAs
// per SM with the tile generator's block loop rolled, and at 3 with it unrolled (the autotuner's
// variants; 2 CTAs lost to 3 and 4 on every measured workload), coupled at the default 2.
template <int MINB, int GU = 1>
static const void* bbu_plain(int model, int pay) {
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_BB_UNI, MOD_GBM, false, MINB, GU>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_BB_UNI, MOD_DUPIRE, false, MINB, GU>(pay);
        case MOD_LVGRID: return pick_payoff<GEN_SOBOL, NOISE_BB_UNI, MOD_LVGRID, false, MINB, GU>(pay);
        default: return nullptr;
    }
}
const void* lookup_sobol_bbu(int model, int pay, bool coupled, int variant) {
    if (coupled) {
        if (variant != 0) return nullptr;
        switch (model) {
            case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_BB_UNI, MOD_GBM, true>(pay);
            case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_BB_UNI, MOD_DUPIRE, true>(pay);
            default: return nullptr;
        }
    }
    switch (variant) {
        case 0: return bbu_plain<3>(model, pay);
        case 1: return bbu_plain<4>(model, pay);
        case 2: return bbu_plain<3, 4>(model, pay);
        default: return nullptr;
    }
}
}  // namespace mcq
