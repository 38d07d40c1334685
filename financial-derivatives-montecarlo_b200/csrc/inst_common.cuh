// inst_common.cuh — helpers for the explicit kernel instantiation units.
#pragma once
#include "path_kernels.cuh"
#include "dispatch.h"

namespace mcq {

template <int GEN, int NOISE, int MOD, bool CPL, int MINB = 0, int GU = 1>
const void* pick_payoff(int pay) {
    switch (pay) {
        case PAY_EUR:
        case PAY_BASKET: return (const void*)&k_pass<GEN, NOISE, PathC<MOD, PAY_EUR, CPL>, MINB, GU>;
        case PAY_ASIAN: return (const void*)&k_pass<GEN, NOISE, PathC<MOD, PAY_ASIAN, CPL>, MINB, GU>;
        case PAY_GEOM: return (const void*)&k_pass<GEN, NOISE, PathC<MOD, PAY_GEOM, CPL>, MINB, GU>;
        case PAY_LOOKBACK: return (const void*)&k_pass<GEN, NOISE, PathC<MOD, PAY_LOOKBACK, CPL>, MINB, GU>;
        case PAY_UPOUT: return (const void*)&k_pass<GEN, NOISE, PathC<MOD, PAY_UPOUT, CPL>, MINB, GU>;
        case PAY_DOWNOUT: return (const void*)&k_pass<GEN, NOISE, PathC<MOD, PAY_DOWNOUT, CPL>, MINB, GU>;
        default: return nullptr;
    }
}

}  // namespace mcq
