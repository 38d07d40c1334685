"""Workloads recorded in ref_golden.npz (shared by make_ref_golden.py and the parity tests)."""
import numpy as np

SALTS = [42, 43, 42 + 16 * 3 + 5, 73]
OFFSETS = [0, 1, (1 << 14) - 1, (1 << 22) - 1, (1 << 32) - (1 << 10)]
DIMS = [(0, 16), (250, 16), (19984, 16)]


def basket_L(n=4, seed=5):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    Cm = A @ A.T + 0.5 * np.eye(n)
    d = np.sqrt(np.diag(Cm))
    return rng, np.linalg.cholesky(Cm / np.outer(d, d))


def cases(T):
    """(name, model, payoff, n_steps, noise, salt0, R, offset, N) with T = the types module."""
    c2m, c2p = T.gbm(100.0, 0.03, 0.25, 1.0), T.asian(100.0)
    hes = T.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    n = 4
    rng, L = basket_L(n)
    return [
        ("asian_raw_256", c2m, c2p, 256, T.RAW, 42, 4, 0, 4096),
        ("asian_bb_256", c2m, c2p, 256, T.BB, 42, 4, 0, 4096),
        ("asian_pca_256", c2m, c2p, 256, T.PCA, 42, 4, 0, 4096),
        ("asian_raw_256_off", c2m, c2p, 256, T.RAW, 300, 2, 12288, 4096),
        ("heston_lookback_64", hes, T.lookback(0.2), 64, T.RAW, 42, 2, 0, 4096),
        ("heston_eur_64", hes, T.european(100.0, 0.02, 1.0), 64, T.RAW, 60, 2, 0, 4096),
        ("dupire_eur_64", T.dupire(100.0, 0.05, 0.2, 0.5, 0.7, 1.0), T.european(100.0, 0.05, 1.0), 64, T.RAW, 42, 2,
         0, 4096),
        ("gbm_upout_64", T.gbm(100.0, 0.05, 0.2, 1.0), T.barrier_up_out(100.0, 125.0, 0.2, 0.05, 1.0), 64, T.RAW, 42,
         2, 0, 4096),
        ("gbm_geom_bb_64", T.gbm(100.0, 0.05, 0.2, 1.0), T.geom_asian(100.0), 64, T.BB, 42, 2, 0, 4096),
        ("basket4_32", T.multi_dupire(100 * rng.uniform(0.8, 1.2, n), L), T.basket(100.0, 0.05, 1.0, n), 32, T.RAW,
         42, 2, 0, 4096),
    ]
