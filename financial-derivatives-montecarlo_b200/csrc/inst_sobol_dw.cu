// Passes on increments computed outside the kernel (NOISE_DW): the large-N PCA route.
#include "inst_common.cuh"
namespace mcq {
const void* lookup_dw(int model, int pay, bool cpl) {
    if (cpl) {
        switch (model) {
            case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_DW, MOD_GBM, true>(pay);
            case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_DW, MOD_DUPIRE, true>(pay);
            default: return nullptr;
        }
    }
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_DW, MOD_GBM, false>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_DW, MOD_DUPIRE, false>(pay);
        case MOD_LVGRID: return pick_payoff<GEN_SOBOL, NOISE_DW, MOD_LVGRID, false>(pay);
        default: return nullptr;
    }
}
}  // namespace mcq
