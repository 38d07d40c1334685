// Drives the caller-side helpers that include/mcq.hpp restates from the reference's utils.cpp,
// with inputs the test controls, and prints what they return (test infrastructure).
//   richardson: estimar_c1_richardson (utils.cpp:174-185) with a deterministic sim_fn
//               P(ns, np, seed) = a + b / ns + c seed, for several (T, M_rich, N_pilot, seed)
//   table:      print_table (utils.cpp:192-210) on fixed rows
#include <cstdio>
#include <string>
#include <vector>

#include "mcq.hpp"

int main(int argc, char** argv) {
    const std::string what = argc > 1 ? argv[1] : "";
    if (what == "richardson") {
        const double a = 10.0, b = 3.0, c = 1e-3;
        auto sim = [&](int ns, long long np, unsigned s) -> double { return a + b / ns + c * s + 0.0 * (double)np; };
        const double Ts[] = {1.0, 0.5, 2.0};
        const int Ms[] = {8, 4, 2};
        for (double T : Ts)
            for (int M : Ms)
                std::printf("%.17g %d %.17g\n", T, M, estimar_c1_richardson(sim, T, M, 50000, 7u));
        // a flat sim_fn: the bias estimate is clamped at 1e-12
        auto flat = [](int, long long, unsigned) -> double { return 1.0; };
        std::printf("flat %.17g\n", estimar_c1_richardson(flat, 1.0, 8, 1000, 0u));
        return 0;
    }
    if (what == "table") {
        std::vector<TableRow> rows = {
            {"MC", 10.4526, 0.00498, 4120904, 0.110},
            {"MLQMC Raw", 10.4504, 0.00033, 141721, 0.637},
            {"QMC PCA", 10.3, 0.012, 1048576, 12.5},
            {"Metodo nombre largo", 99.123456, 1.5, 12345678901LL, 1234.5678},
        };
        print_table(rows, 10.450584, 0.05, "Ejemplo de prueba");
        return 0;
    }
    return 2;
}
