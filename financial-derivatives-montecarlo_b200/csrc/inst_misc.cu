#include "inst_common.cuh"
namespace mcq {

template <int GEN>
static const void* misc_gen(int noise, int est, int model, int nb, bool dump) {
    if (dump) {
        if (noise == NOISE_RAW) return (const void*)&k_pass<GEN, NOISE_RAW, DumpC>;
        if (noise == NOISE_BB && GEN == GEN_SOBOL) return (const void*)&k_pass<GEN_SOBOL, NOISE_BB, DumpC>;
        if (noise == NOISE_PCA && GEN == GEN_SOBOL) return (const void*)&k_pass<GEN_SOBOL, NOISE_PCA, DumpC>;
        return nullptr;
    }
    if (noise != NOISE_RAW) return nullptr;
    if (est == EST_CV_ASIAN) return (const void*)&k_pass<GEN, NOISE_RAW, CvAsianC>;
    if (est == EST_CV_DUPIRE) return (const void*)&k_pass<GEN, NOISE_RAW, CvDupireC>;
    if (est == EST_IS) return (const void*)&k_pass<GEN, NOISE_RAW, IsC>;
    if (est == EST_COUPLED && model == MOD_BASKET) {
        if (nb <= 4) return (const void*)&k_pass<GEN, NOISE_RAW, BasketLevelC<MOD_BASKET, 4>>;
        if (nb <= 8) return (const void*)&k_pass<GEN, NOISE_RAW, BasketLevelC<MOD_BASKET, 8>, 2>;
        if (nb <= 16) return (const void*)&k_pass<GEN, NOISE_RAW, BasketLevelC<MOD_BASKET, 16>, 1>;
        return nullptr;
    }
    if (est == EST_COUPLED && model == MOD_MULTI) {
        if (nb <= 4) return (const void*)&k_pass<GEN, NOISE_RAW, BasketLevelC<MOD_MULTI, 4>>;
        if (nb <= 8) return (const void*)&k_pass<GEN, NOISE_RAW, BasketLevelC<MOD_MULTI, 8>, 2>;
        if (nb <= 16) return (const void*)&k_pass<GEN, NOISE_RAW, BasketLevelC<MOD_MULTI, 16>, 1>;
        return nullptr;
    }
    if (model == MOD_MULTI) {
        if (nb <= 4) return (const void*)&k_pass<GEN, NOISE_RAW, BasketC<MOD_MULTI, 4>>;
        if (nb <= 8) return (const void*)&k_pass<GEN, NOISE_RAW, BasketC<MOD_MULTI, 8>>;
        if (nb <= 16) return (const void*)&k_pass<GEN, NOISE_RAW, BasketC<MOD_MULTI, 16>>;
        if (nb <= kMaxWideBasket) return (const void*)&k_pass<GEN, NOISE_RAW, BasketWideC<MOD_MULTI>>;
        if (nb <= kMaxHugeBasket) return (const void*)&k_pass<GEN, NOISE_RAW, BasketWideC<MOD_MULTI, kMaxHugeBasket>>;
        return nullptr;
    }
    if (model == MOD_BASKET) {
        if (nb <= 4) return (const void*)&k_pass<GEN, NOISE_RAW, BasketC<MOD_BASKET, 4>>;
        if (nb <= 8) return (const void*)&k_pass<GEN, NOISE_RAW, BasketC<MOD_BASKET, 8>>;
        if (nb <= 16) return (const void*)&k_pass<GEN, NOISE_RAW, BasketC<MOD_BASKET, 16>>;
        if (nb <= kMaxWideBasket) return (const void*)&k_pass<GEN, NOISE_RAW, BasketWideC<MOD_BASKET>>;
        if (nb <= kMaxHugeBasket) return (const void*)&k_pass<GEN, NOISE_RAW, BasketWideC<MOD_BASKET, kMaxHugeBasket>>;
        return nullptr;
    }
    return nullptr;
}

const void* lookup_misc(int gen, int noise, int est, int model, int nb, bool dump) {
    return gen == GEN_SOBOL ? misc_gen<GEN_SOBOL>(noise, est, model, nb, dump)
                            : misc_gen<GEN_PHILOX>(noise, est, model, nb, dump);
}
}  // namespace mcq
