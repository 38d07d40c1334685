#include "inst_common.cuh"
namespace mcq {
const void* lookup_philox_plain(int model, int pay) {
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN_PHILOX, NOISE_RAW, MOD_GBM, false>(pay);
        case MOD_HESTON: return pick_payoff<GEN_PHILOX, NOISE_RAW, MOD_HESTON, false>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN_PHILOX, NOISE_RAW, MOD_DUPIRE, false>(pay);
        case MOD_LVGRID: return pick_payoff<GEN_PHILOX, NOISE_RAW, MOD_LVGRID, false>(pay);
        default: return nullptr;
    }
}
}  // namespace mcq
