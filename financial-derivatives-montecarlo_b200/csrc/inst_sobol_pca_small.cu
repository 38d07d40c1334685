// Single-tile PCA passes (N <= 32 steps): coarse MLQMC levels and short products.
#include "inst_common.cuh"
namespace mcq {
const void* lookup_sobol_pca_small(int model, int pay, bool cpl) {
    if (cpl) {
        switch (model) {
            case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_PCA, MOD_GBM, true>(pay);
            case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_PCA, MOD_DUPIRE, true>(pay);
            default: return nullptr;
        }
    }
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_SOBOL, NOISE_PCA, MOD_GBM, false>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_SOBOL, NOISE_PCA, MOD_DUPIRE, false>(pay);
        case MOD_LVGRID: return pick_payoff<GEN_SOBOL, NOISE_PCA, MOD_LVGRID, false>(pay);
        default: return nullptr;
    }
}
}  // namespace mcq
