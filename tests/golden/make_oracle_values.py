#!/usr/bin/env python
"""FP64 oracle values for every workload the benchmark prices, written to oracle_values.json.

Each benchmark result states its error against these (bench.py reads the JSON; nothing here
runs on the GPU).  What each value is:

  mc_gbm_european        Black–Scholes closed form (S0 = K = 100, r = 0.05, sigma = 0.2, T = 1).
  asian_gbm_256          arithmetic-average Asian call, GBM S0 = K = 100, r = 0.03, sigma = 0.25,
                         T = 1, 256 Euler steps: FP64 oracle RQMC over 32 replicas x 2^22 scrambled
                         Sobol points with salts 1042.. (independent of the engine's 42..), the
                         same discretisation as the engine; plus the discrete geometric-Asian
                         closed form of the same contract (the geometric check pass).
  mlqmc_heston_*         Heston (kappa 2, theta 0.04, xi 0.3, rho -0.7, v0 0.04, S0 100, r 0.02,
                         T 1) with the Euler–Milstein variance step, lookback (BGK sigma 0.2) and
                         down-and-out call (K 100, B 80): the FP64 oracle's MLQMC driver
                         (oracle_py.run_mlqmc, the arithmetic of run_mlqmc_cuda) at eps = 5e-4,
                         M = 4, 4 steps on level 0, L <= 8, R = 16, salts 1042...
  asian_gbm_256_engine_points  the same contract's FP64 per-replica sums on the benchmark pass's own
                         points (salts 42.., 32 x 2^20), for a same-points check of the full-size pass.
  adjoint_localvol_asian the adjoint workload (64 x 32 local-vol grid, Asian call, T = 2, 512
                         steps): price from FP64 oracle RQMC over 16 x 2^20 independent points
                         (salts 1042..); delta, rho and vega (parallel shift of the grid) as FP64
                         central differences of the oracle on the engine's own points (salts
                         42.., 16 x 2^18 points, h = 1e-4 relative).
  book                   a sample of the synthetic basket book (seed 5): FP64 oracle MLQMC of the
                         coupled basket pair (orc_basket_level_sums) at eps = 5e-4 (the options'
                         own M = 2, n0 = 1, max_L, R = 16, salts 1042..), price and per-asset
                         deltas.  One-asset options of the book are checked against Black–Scholes
                         by the benchmark itself.

Usage: python tests/golden/make_oracle_values.py [--only KEY ...] [--book-sample N]
The file is updated key by key, so an interrupted run keeps what it finished.
"""
import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "oracle_values.json")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle_py as orc  # noqa: E402

T = orc.T
SALT = 1042


def load():
    try:
        with open(OUT) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save(d):
    with open(OUT + ".tmp", "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(OUT + ".tmp", OUT)


def mc_gbm_european():
    return {"value": orc.bs_call(100.0, 100.0, 1.0, 0.05, 0.2), "se": 0.0,
            "kind": "Black-Scholes closed form"}


def asian_gbm_256():
    m, p = T.gbm(100.0, 0.03, 0.25, 1.0), T.asian(100.0)
    R, N = 32, 1 << 22
    s = orc.qmc_sums(m, p, 256, None, SALT, R, 0, N)
    rm = s[:, 0] / N
    return {"value": float(rm.mean()), "se": float(rm.std(ddof=1) / np.sqrt(R)),
            "kind": f"FP64 oracle RQMC, {R} replicas x 2^22 points, 256 Euler steps, salts {SALT}..",
            "geom_closed_form": orc.geom_asian(100.0, 100.0, 1.0, 0.03, 0.25, 256)}


def asian_engine_points():
    """FP64 per-replica sums on the benchmark pass's own points (salts 42.., 2^20 points per replica):
    the engine's full-size pass is checked against them replica by replica."""
    m, p = T.gbm(100.0, 0.03, 0.25, 1.0), T.asian(100.0)
    R, N = 32, 1 << 20
    s = orc.qmc_sums(m, p, 256, None, 42, R, 0, N)
    return {"sums": s.tolist(), "R": R, "N": N, "salt_base": 42,
            "kind": "FP64 oracle per-replica {sum Y, sum Y^2}, the bench pass's points (salts 42.., 2^20 per replica)"}


def heston(pay):
    m = T.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    p = T.lookback(0.2) if pay == "lookback" else T.barrier_down_out(100.0, 80.0, 0.2, 0.02, 1.0)
    r = orc.run_mlqmc(m, p, 5e-4, M=4, max_L=8, n0=4, R=16, salt_base=SALT, flags=T.FLAG_HESTON_MILSTEIN)
    return {"value": float(r["price"]), "se": float(r["std_error"]), "levels": int(r["levels"]),
            "converged": bool(r["converged"]),
            "kind": f"FP64 oracle MLQMC eps=5e-4, M=4, n0=4, L<=8, R=16, Euler-Milstein variance, salts {SALT}.."}


def adjoint_localvol():
    K, t, g = T.config4_surface()
    build = lambda S0=100.0, mu=0.05, shift=0.0: T.localvol_grid(K, t, g + shift, S0, mu, 2.0)   # noqa: E731
    p = T.asian(100.0)
    n = 512
    R, N = 16, 1 << 20
    s = orc.qmc_sums(build(), p, n, None, SALT, R, 0, N)
    rm = s[:, 0] / N

    def price(m):
        q = orc.qmc_sums(m, p, n, None, 42, 16, 0, 1 << 18)
        return q[:, 0].sum() / (16 << 18)

    h = 1e-4
    delta = (price(build(S0=100.0 * (1 + h))) - price(build(S0=100.0 * (1 - h)))) / (2 * 100.0 * h)
    rho = (price(build(mu=0.05 * (1 + h))) - price(build(mu=0.05 * (1 - h)))) / (2 * 0.05 * h)
    vega = (price(build(shift=0.2 * h)) - price(build(shift=-0.2 * h))) / (2 * 0.2 * h)
    return {"price": float(rm.mean()), "price_se": float(rm.std(ddof=1) / np.sqrt(R)),
            "delta": float(delta), "rho": float(rho), "vega": float(vega),
            "kind": f"price: FP64 oracle RQMC 16 x 2^20 points, salts {SALT}..; delta / rho / vega: FP64 "
                    "central differences (h = 1e-4 relative; vega = parallel shift of the grid) on the "
                    "engine's points (salts 42.., 16 x 2^18)"}


def book_sample(n_sample):
    book = T.config5_book(n=4096, seed=5)
    out = {}
    idx = [i for i in range(len(book)) if book[i].n_assets >= 2][:n_sample]
    for i in idx:
        o = book[i]
        d = o.n_assets
        S0 = np.ctypeslib.as_array(o.S0, (d,)).copy()
        sig = np.ctypeslib.as_array(o.sigma, (d,)).copy()
        w = np.ctypeslib.as_array(o.weights, (d,)).copy()
        L = np.ctypeslib.as_array(o.L, (d * d,)).copy().reshape(d, d)
        m = T.basket_gbm(S0, sig, L=L, weights=w, mu=o.r, T=o.T)
        p = T.basket(o.K, o.r, o.T, d)
        t0 = time.time()
        r = orc.run_mlqmc(m, p, 5e-4, M=2, max_L=o.max_L, n0=1, R=16, salt_base=SALT, basket=True)
        out[str(i)] = {"value": float(r["price"]), "se": float(r["std_error"]), "levels": int(r["levels"]),
                       "converged": bool(r["converged"]), "delta": [float(x) for x in r["delta"]],
                       "assets": d, "seconds": time.time() - t0}
        print("book option", i, out[str(i)], flush=True)
    return {"options": out,
            "kind": f"FP64 oracle MLQMC of the coupled basket pair, eps=5e-4, M=2, n0=1, the option's max_L, "
                    f"R=16, salts {SALT}..; first {n_sample} options of the seed-5 book with >= 2 assets"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=None)
    ap.add_argument("--book-sample", type=int, default=4)
    a = ap.parse_args()
    jobs = [("mc_gbm_european", mc_gbm_european), ("asian_gbm_256", asian_gbm_256),
            ("asian_gbm_256_engine_points", asian_engine_points),
            ("adjoint_localvol_asian", adjoint_localvol),
            ("mlqmc_heston_lookback", lambda: heston("lookback")),
            ("mlqmc_heston_down_out", lambda: heston("down_out")),
            ("book", lambda: book_sample(a.book_sample))]
    d = load()
    for key, fn in jobs:
        if a.only is not None and key not in a.only:
            continue
        t0 = time.time()
        d[key] = fn()
        d[key]["generated_s"] = round(time.time() - t0, 1)
        save(d)
        print(key, d[key], flush=True)


if __name__ == "__main__":
    main()
