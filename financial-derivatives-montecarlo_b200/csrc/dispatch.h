// dispatch.h — lookup of the fused pass kernel instantiated for a (generator, noise, estimator,
// model, payoff) combination.  The instantiations are spread over several translation units
// so that they compile in parallel; each returns nullptr for a combination it does not hold.
#pragma once
#include "kparams.h"

namespace mcq {

const void* lookup_sobol_raw_plain(int model, int payoff);
const void* lookup_sobol_raw_plain_b4(int model, int payoff);   // 64-register variant
const void* lookup_sobol_raw_plain_u4(int model, int payoff);   // 64 registers, unrolled tile
const void* lookup_sobol_raw_coupled(int model, int payoff);
const void* lookup_sobol_raw_coupled_b4(int model, int payoff);   // 64-register variant
const void* lookup_sobol_raw_coupled_u4(int model, int payoff);   // 64 registers, unrolled tile
const void* lookup_sobol_packed(int model, int payoff, bool coupled);   // raw, D <= 16 (NOISE_PACKED)
const void* lookup_assist(int gen, int model, int payoff, bool coupled);  // raw, few long paths (NOISE_ASSIST)
const void* lookup_sobol_bb(int model, int payoff, bool coupled);
const void* lookup_sobol_bb_b3(int model, int payoff);          // 3-CTA (80-register) variant
const void* lookup_sobol_bbu(int model, int payoff, bool coupled, int variant);   // NOISE_BB_UNI
const void* lookup_sobol_pca_small(int model, int payoff, bool coupled);   // N <= 32
const void* lookup_dw(int model, int payoff, bool coupled);   // NOISE_DW (large-N PCA increments)
const void* lookup_philox_plain(int model, int payoff);
const void* lookup_philox_coupled(int model, int payoff);
// est in {EST_CV_ASIAN, EST_CV_DUPIRE, EST_IS}, basket models (nb = 4, 8, 16), dump probes
const void* lookup_misc(int gen, int noise, int est, int model, int nb, bool dump);

// Kernel families with more than one compiled launch variant (see the autotuner in engine.cpp).
inline int n_variants(int gen, int noise, int est, int model) {
    if (gen != GEN_SOBOL || model == MOD_MULTI || model == MOD_BASKET) return 1;
    if (est == EST_COUPLED) return (noise == NOISE_RAW && model != MOD_LVGRID) ? 3 : 1;
    if (est != EST_PLAIN) return 1;
    if (noise == NOISE_RAW) return 3;
    if (noise == NOISE_BB && model != MOD_HESTON) return 2;
    if (noise == NOISE_BB_UNI && model != MOD_HESTON) return 3;
    return 1;
}
inline const void* lookup_variant(int gen, int noise, int est, int model, int payoff, int variant) {
    if (variant < 1 || variant >= n_variants(gen, noise, est, model)) return nullptr;
    if (est == EST_COUPLED)
        return variant == 1 ? lookup_sobol_raw_coupled_b4(model, payoff) : lookup_sobol_raw_coupled_u4(model, payoff);
    if (noise == NOISE_BB_UNI) return lookup_sobol_bbu(model, payoff, false, variant);
    if (noise == NOISE_RAW)
        return variant == 1 ? lookup_sobol_raw_plain_b4(model, payoff) : lookup_sobol_raw_plain_u4(model, payoff);
    return lookup_sobol_bb_b3(model, payoff);
}

inline const void* lookup_pass(int gen, int noise, int est, int model, int payoff, int nb) {
    if (model == MOD_MULTI || model == MOD_BASKET || est >= EST_CV_ASIAN)
        return lookup_misc(gen, noise, est, model, nb, false);
    const bool cpl = (est == EST_COUPLED);
    if (gen == GEN_SOBOL) {
        if (noise == NOISE_RAW) return cpl ? lookup_sobol_raw_coupled(model, payoff) : lookup_sobol_raw_plain(model, payoff);
        if (noise == NOISE_BB) return lookup_sobol_bb(model, payoff, cpl);
        if (noise == NOISE_BB_UNI) return lookup_sobol_bbu(model, payoff, cpl, 0);
        if (noise == NOISE_PCA) return lookup_sobol_pca_small(model, payoff, cpl);
        return nullptr;
    }
    if (noise != NOISE_RAW) return nullptr;
    return cpl ? lookup_philox_coupled(model, payoff) : lookup_philox_plain(model, payoff);
}

}  // namespace mcq
