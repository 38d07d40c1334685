#include "inst_common.cuh"
namespace mcq {
const void* lookup_philox_coupled(int model, int pay) {
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_PHILOX, NOISE_RAW, MOD_GBM, true>(pay);
        case MOD_HESTON: return pick_payoff<GEN_PHILOX, NOISE_RAW, MOD_HESTON, true>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_PHILOX, NOISE_RAW, MOD_DUPIRE, true>(pay);
        default: return nullptr;
    }
}
}  // namespace mcq
