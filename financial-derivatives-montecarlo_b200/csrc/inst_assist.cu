#include "inst_common.cuh"
namespace mcq {
// Raw-ordered passes with few, long paths (NOISE_ASSIST): Sobol and Philox, plain and coupled.
template <int GEN>
static const void* assist_models(int model, int pay, bool coupled) {
    if (coupled) {
        switch (model) {
            case MOD_GBM: return pick_payoff<GEN, NOISE_ASSIST, MOD_GBM, true>(pay);
            case MOD_HESTON: return pick_payoff<GEN, NOISE_ASSIST, MOD_HESTON, true>(pay);
            case MOD_DUPIRE: return pick_payoff<GEN, NOISE_ASSIST, MOD_DUPIRE, true>(pay);
            default: return nullptr;
        }
    }
    switch (model) {
        case MOD_GBM: return pick_payoff<GEN, NOISE_ASSIST, MOD_GBM, false>(pay);
        case MOD_HESTON: return pick_payoff<GEN, NOISE_ASSIST, MOD_HESTON, false>(pay);
        case MOD_DUPIRE: return pick_payoff<GEN, NOISE_ASSIST, MOD_DUPIRE, false>(pay);
        case MOD_LVGRID: return pick_payoff<GEN, NOISE_ASSIST, MOD_LVGRID, false>(pay);
        default: return nullptr;
    }
}
const void* lookup_assist(int gen, int model, int pay, bool coupled) {
    return gen == GEN_SOBOL ? assist_models<GEN_SOBOL>(model, pay, coupled)
                            : assist_models<GEN_PHILOX>(model, pay, coupled);
}
}  // namespace mcq
