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


def level_cases(T):
    """Coupled level passes of the reference's kernel_mlmc (methods_cuda.cu:445-518), n0 = 1 as the
    reference (N_fine = M^l): (name, model, payoff, level, M, salt0, R, offset, N).  The recorded
    salt may be moved by make_ref_golden.py off a window with a u = 1 point."""
    gbm, hes = T.gbm(100.0, 0.05, 0.2, 1.0), T.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    dup = T.dupire(100.0, 0.05, 0.2, 0.5, 0.7, 1.0)
    out = []
    for lv in range(4):
        out.append((f"lvl_gbm_eur_M4_l{lv}", gbm, T.european(100.0, 0.05, 1.0), lv, 4, 500 + lv, 2, 0, 4096))
        out.append((f"lvl_heston_eur_M4_l{lv}", hes, T.european(100.0, 0.02, 1.0), lv, 4, 520 + lv, 2, 0, 4096))
        out.append((f"lvl_dupire_eur_M2_l{lv}", dup, T.european(100.0, 0.05, 1.0), lv, 2, 540 + lv, 2, 0, 4096))
    for lv in (1, 3):
        out.append((f"lvl_gbm_asian_M2_l{lv}", gbm, T.asian(100.0), lv, 2, 560 + lv, 2, 64, 4096))
        out.append((f"lvl_gbm_lookback_M4_l{lv}", gbm, T.lookback(0.2), lv, 4, 580 + lv, 2, 0, 4096))
        # the reference's Heston level kernel skips the running update (trap of :464-490): the
        # engine matches it under MCQ_FLAG_COMPAT_HESTON_MLMC
        out.append((f"lvl_heston_lookback_M4_l{lv}", hes, T.lookback(0.2), lv, 4, 600 + lv, 2, 0, 4096))
    out.append(("lvl_gbm_upout_M4_l2", gbm, T.barrier_up_out(100.0, 125.0, 0.2, 0.05, 1.0), 2, 4, 620, 2, 0, 4096))
    return out


def is_cases(T):
    """kernel_is_gbm (methods_cuda.cu:685-707) on scrambled Sobol normals:
    (name, model, payoff, n_steps, z_star (whole path; the kernel takes z_star / sqrt(n_steps)),
    salt0, R, offset, N)."""
    gbm = T.gbm(100.0, 0.05, 0.2, 1.0)
    return [
        ("is_atm_64", gbm, T.european(100.0, 0.05, 1.0), 64, 0.5, 700, 2, 0, 4096),
        ("is_otm180_100", gbm, T.european(180.0, 0.05, 1.0), 100, 3.0, 710, 2, 0, 4096),
        ("is_otm180_100_off", gbm, T.european(180.0, 0.05, 1.0), 100, 3.0, 720, 2, 8192, 4096),
    ]
