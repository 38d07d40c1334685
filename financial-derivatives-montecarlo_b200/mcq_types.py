"""ctypes mirrors of the structs in include/mcq.h, plus builders for models and payoffs.

This module only describes data; it loads no library.  The engine binding (this package's
__init__) and the test oracle binding both use it.
"""
import ctypes as C

import numpy as np

# model / payoff / noise enumerations (include/mcq.h)
GBM, HESTON, DUPIRE, MULTI_DUPIRE, LOCALVOL_GRID, BASKET_GBM = range(6)
EUROPEAN, ASIAN, GEOM_ASIAN, LOOKBACK, BARRIER_UP_OUT, BASKET, BARRIER_DOWN_OUT = range(7)
RAW, BB, PCA = range(3)
FLAG_COMPAT_U_INF = 1
FLAG_COMPAT_HESTON_MLMC = 2
FLAG_HESTON_MILSTEIN = 8
FLAG_BASKET_OWN_S0 = 16

_pd = C.POINTER(C.c_double)


class Model(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("n_assets", C.c_int32),
        ("S0", C.c_double), ("mu", C.c_double), ("T", C.c_double),
        ("sigma", C.c_double),
        ("kappa", C.c_double), ("theta", C.c_double), ("xi", C.c_double), ("rho", C.c_double),
        ("v0", C.c_double), ("hes_L10", C.c_double), ("hes_L11", C.c_double),
        ("sigma0", C.c_double), ("alpha", C.c_double), ("beta_d", C.c_double),
        ("uncorrelated", C.c_int32), ("_pad0", C.c_int32),
        ("S0_vec", _pd), ("L", _pd), ("sigma_vec", _pd), ("weights", _pd),
        ("lv_nK", C.c_int32), ("lv_nt", C.c_int32),
        ("lv_K", _pd), ("lv_t", _pd), ("lv_sigma", _pd),
    ]


class Payoff(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_assets", C.c_int32), ("K", C.c_double), ("B", C.c_double),
                ("r", C.c_double), ("T", C.c_double), ("sigma", C.c_double)]


class MCCfg(C.Structure):
    _fields_ = [("N_batch", C.c_int64), ("pilot_n", C.c_int32), ("seed", C.c_uint32)]


class QMCCfg(C.Structure):
    _fields_ = [("R", C.c_int32), ("max_doublings", C.c_int32), ("N0_per_replica", C.c_int64),
                ("salt_base", C.c_uint32), ("flags", C.c_int32)]


class MLMCCfg(C.Structure):
    _fields_ = [("M", C.c_int32), ("max_L", C.c_int32), ("pilot_n", C.c_int32), ("n0_steps", C.c_int32),
                ("flags", C.c_int32), ("seed", C.c_uint32)]


class Result(C.Structure):
    _fields_ = [("price", C.c_double), ("std_error", C.c_double), ("n_samples", C.c_int64),
                ("time_s", C.c_double), ("path_steps", C.c_double), ("levels", C.c_int32),
                ("launches", C.c_int32), ("converged", C.c_int32), ("reserved", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Greeks(C.Structure):
    _fields_ = [("price", C.c_double), ("delta", C.c_double), ("rho", C.c_double), ("vega", C.c_double),
                ("price_se", C.c_double), ("delta_se", C.c_double), ("rho_se", C.c_double),
                ("vega_se", C.c_double), ("n_paths", C.c_int64), ("n_nodes", C.c_int32),
                ("launches", C.c_int32), ("time_s", C.c_double), ("path_steps", C.c_double)]


BOOK_MAX_ASSETS = 16
BOOK_BATCHED, BOOK_PLAIN = 0, 1


class BookOption(C.Structure):
    _fields_ = [("n_assets", C.c_int32), ("max_L", C.c_int32), ("K", C.c_double), ("r", C.c_double),
                ("T", C.c_double), ("eps", C.c_double), ("S0", _pd), ("sigma", _pd), ("weights", _pd),
                ("L", _pd), ("model", C.POINTER(Model)), ("payoff", C.POINTER(Payoff))]


class BookResult(C.Structure):
    _fields_ = [("price", C.c_double), ("std_error", C.c_double), ("delta", C.c_double * BOOK_MAX_ASSETS),
                ("n_samples", C.c_int64), ("levels", C.c_int32), ("converged", C.c_int32)]


class BookStats(C.Structure):
    _fields_ = [("time_s", C.c_double), ("setup_s", C.c_double), ("path_steps", C.c_double),
                ("normals", C.c_double), ("rounds", C.c_int32), ("launches", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class CVPilotOut(C.Structure):
    _fields_ = [("beta", C.c_double), ("var_plain", C.c_double), ("var_cv", C.c_double)]


def _arr(x):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    return a, a.ctypes.data_as(_pd)


def _keep(m, *arrays):
    m._keep = getattr(m, "_keep", []) + list(arrays)
    return m


def gbm(S0=100.0, mu=0.05, sigma=0.2, T=1.0):
    m = Model()
    m.kind, m.S0, m.mu, m.sigma, m.T = GBM, S0, mu, sigma, T
    return m


def heston(S0=100.0, mu=0.05, kappa=2.0, theta=0.04, xi=0.5, rho=-0.9, v0=0.04, T=1.0):
    m = Model()
    m.kind, m.S0, m.mu, m.kappa, m.theta, m.xi, m.rho, m.v0, m.T = HESTON, S0, mu, kappa, theta, xi, rho, v0, T
    m.hes_L10, m.hes_L11 = rho, float(np.sqrt(1.0 - rho * rho))
    return m


def dupire(S0=100.0, mu=0.05, sigma0=0.2, alpha=0.5, beta_d=0.7, T=1.0):
    m = Model()
    m.kind, m.S0, m.mu, m.sigma0, m.alpha, m.beta_d, m.T = DUPIRE, S0, mu, sigma0, alpha, beta_d, T
    m.sigma = sigma0
    return m


def multi_dupire(S0_vec, L=None, mu=0.05, sigma0=0.2, alpha=0.5, beta_d=0.7, T=1.0):
    m = Model()
    s, ps = _arr(S0_vec)
    m.kind, m.n_assets, m.mu, m.sigma0, m.alpha, m.beta_d, m.T = MULTI_DUPIRE, len(s), mu, sigma0, alpha, beta_d, T
    m.S0, m.S0_vec = float(s[0]), ps
    keep = [s]
    if L is None:
        m.uncorrelated = 1
    else:
        la, pl = _arr(L)
        m.L = pl
        keep.append(la)
    return _keep(m, *keep)


def basket_gbm(S0_vec, sigma_vec, L=None, weights=None, mu=0.05, T=1.0):
    m = Model()
    s, ps = _arr(S0_vec)
    sg, psg = _arr(sigma_vec)
    m.kind, m.n_assets, m.mu, m.T = BASKET_GBM, len(s), mu, T
    m.S0, m.S0_vec, m.sigma_vec = float(s[0]), ps, psg
    keep = [s, sg]
    if L is None:
        m.uncorrelated = 1
    else:
        la, pl = _arr(L)
        m.L = pl
        keep.append(la)
    if weights is not None:
        w, pw = _arr(weights)
        m.weights = pw
        keep.append(w)
    return _keep(m, *keep)


def config4_surface(seed=4, noise_sd=0.01):
    """The local-vol surface of the adjoint workload: 64 strikes in [50, 150] x 32 times in [0, 2],
    sigma(K, t) = 0.2 + 0.1 exp(-(K/100 - 1)^2 / 0.05) (1 + 0.5 t) plus seeded N(0, noise_sd^2)
    noise (noise_sd read as the standard deviation), clipped below at 0.05."""
    K = np.linspace(50.0, 150.0, 64)
    t = np.linspace(0.0, 2.0, 32)
    g = 0.2 + 0.1 * np.exp(-(K[None, :] / 100.0 - 1.0) ** 2 / 0.05) * (1.0 + 0.5 * t[:, None])
    g = g + np.random.default_rng(seed).normal(0.0, noise_sd, g.shape)
    return K, t, np.maximum(g, 0.05)


def book_option(S0, sigma, K, r, T, eps, max_L, weights=None, L=None):
    """One basket call of a book: max(sum_a w_a S_a(T) - K, 0) e^{-rT} on correlated GBM assets
    (L: lower Cholesky factor of the correlation, row-major; None: uncorrelated)."""
    o = BookOption()
    s0, p0 = _arr(S0)
    sg, ps = _arr(sigma)
    d = len(s0)
    keep = [s0, sg]
    o.n_assets, o.max_L, o.K, o.r, o.T, o.eps = d, int(max_L), K, r, T, eps
    o.S0, o.sigma = p0, ps
    if weights is not None:
        w, pw = _arr(weights)
        o.weights = pw
        keep.append(w)
    if L is not None:
        l, pl = _arr(np.asarray(L, dtype=np.float64).reshape(d, d))
        o.L = pl
        keep.append(l)
    return _keep(o, *keep)


def book_single(model, payoff, eps, max_L):
    """A single-asset option of a book: `model` (GBM, Heston, parametric Dupire) with `payoff`,
    priced by MLQMC to eps with levels up to max_L (no deltas)."""
    o = BookOption()
    o.n_assets, o.max_L, o.eps, o.T = 1, int(max_L), eps, model.T
    o.model, o.payoff = C.pointer(model), C.pointer(payoff)
    return _keep(o, model, payoff)


def mixed_singles(n=256, seed=6, r=0.02):
    """Single-asset options for a mixed book: models GBM (sigma ~ U[0.1, 0.4]), Heston (the
    benchmark's Heston parameters with xi ~ U[0.2, 0.5], rho ~ U[-0.8, -0.3]) and parametric Dupire
    (sigma0 ~ U[0.15, 0.3]) in turn, S0 100, T ~ U[0.25, 2], with European, Asian, lookback and
    down-and-out (B = 80) payoffs in turn (Dupire options take the down-and-out call in place of the
    lookback: on the coarsest levels an Euler step spans up to T, a path can step below 0, and the
    local volatility (S / S0)^(beta - 1) is then NaN, which the lookback's S_T - min S carries into
    the price as the reference's formulas do), K = 100 U[0.9, 1.1], eps ~ U[5e-4, 5e-3] and
    max_L 6 (M = 2, n0 = 1: 64 finest steps)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        T = float(rng.uniform(0.25, 2.0))
        kind = i % 3
        if kind == 0:
            m = gbm(100.0, r, float(rng.uniform(0.1, 0.4)), T)
        elif kind == 1:
            m = heston(100.0, r, 2.0, 0.04, float(rng.uniform(0.2, 0.5)), float(rng.uniform(-0.8, -0.3)), 0.04, T)
        else:
            m = dupire(100.0, r, float(rng.uniform(0.15, 0.3)), 0.5, 0.7, T)
        K = float(100.0 * rng.uniform(0.9, 1.1))
        pk = (i // 3) % 4
        if kind == 2 and pk == 2:
            pk = 3
        p = (european(K, r, T), asian(K), lookback(0.2), barrier_down_out(K, 80.0, 0.2, r, T))[pk]
        out.append(book_single(m, p, float(rng.uniform(5e-4, 5e-3)), 6))
    return out


def config5_book(n=4096, seed=5, r=0.03):
    """The batched heterogeneous book: n basket calls, d ~ U{1..16}, S0_i = 100 U[0.8, 1.2],
    sigma_i ~ U[0.1, 0.5], correlation from a seeded A A^T + 0.5 I normalised to unit diagonal
    (its Cholesky factor is passed), weights ~ Dirichlet(1), K = U[0.8, 1.2] x the weighted
    forward, T ~ U[0.1, 3], 2^k steps with k ~ U{4..9} on the finest level (n0 = 1, M = 2, so
    max_L = k), eps ~ U[5e-4, 5e-3].  r is common to the book (the workload leaves it open)."""
    rng = np.random.default_rng(seed)
    book = []
    for _ in range(n):
        d = int(rng.integers(1, 17))
        S0 = 100.0 * rng.uniform(0.8, 1.2, d)
        sig = rng.uniform(0.1, 0.5, d)
        A = rng.normal(size=(d, d))
        Cm = A @ A.T + 0.5 * np.eye(d)
        dg = np.sqrt(np.diag(Cm))
        corr = Cm / np.outer(dg, dg)
        L = np.linalg.cholesky(corr)
        w = rng.dirichlet(np.ones(d))
        T = float(rng.uniform(0.1, 3.0))
        K = float(rng.uniform(0.8, 1.2) * np.dot(w, S0) * np.exp(r * T))
        k = int(rng.integers(4, 10))
        eps = float(rng.uniform(5e-4, 5e-3))
        book.append(book_option(S0, sig, K, r, T, eps, k, weights=w, L=L))
    return book


def localvol_grid(K_axis, t_axis, sigma_grid, S0=100.0, mu=0.05, T=1.0):
    """sigma_grid[j, i] = sigma(K_i, t_j)."""
    m = Model()
    k, pk = _arr(K_axis)
    t, pt = _arr(t_axis)
    g, pg = _arr(np.asarray(sigma_grid, dtype=np.float64).reshape(len(t), len(k)))
    m.kind, m.S0, m.mu, m.T = LOCALVOL_GRID, S0, mu, T
    m.lv_nK, m.lv_nt, m.lv_K, m.lv_t, m.lv_sigma = len(k), len(t), pk, pt, pg
    return _keep(m, k, t, g)


def payoff(kind, K=100.0, B=0.0, r=0.05, T=1.0, sigma=0.2, n_assets=0):
    p = Payoff()
    p.kind, p.K, p.B, p.r, p.T, p.sigma, p.n_assets = kind, K, B, r, T, sigma, n_assets
    return p


def european(K, r, T):
    return payoff(EUROPEAN, K=K, r=r, T=T)


def asian(K):
    return payoff(ASIAN, K=K)


def geom_asian(K):
    return payoff(GEOM_ASIAN, K=K)


def lookback(sigma):
    return payoff(LOOKBACK, sigma=sigma)


def barrier_up_out(K, B, sigma, r, T):
    return payoff(BARRIER_UP_OUT, K=K, B=B, sigma=sigma, r=r, T=T)


def barrier_down_out(K, B, sigma, r, T):
    return payoff(BARRIER_DOWN_OUT, K=K, B=B, sigma=sigma, r=r, T=T)


def basket(K, r, T, n_assets):
    return payoff(BASKET, K=K, r=r, T=T, n_assets=n_assets)


def noise_dim(m):
    if m.kind == HESTON:
        return 2
    if m.kind in (MULTI_DUPIRE, BASKET_GBM):
        return m.n_assets
    return 1
