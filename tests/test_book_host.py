"""Batched book, host side (no GPU): argument checks through the C ABI, the synthetic book's
distributions, and the oracle's coupled basket pair and its pathwise delta against FP64
finite differences."""
import ctypes as C

import numpy as np
import pytest


def _one(eng, d=3, max_L=4, **kw):
    rng = np.random.default_rng(1)
    S0 = 100 * rng.uniform(0.8, 1.2, d)
    sig = rng.uniform(0.1, 0.5, d)
    args = dict(K=100.0, r=0.03, T=1.0, eps=1e-2, max_L=max_L)
    args.update(kw)
    return eng.book_option(S0, sig, **args)


def test_book_rejects_bad_input_before_touching_the_gpu(eng):
    L = eng.lib()
    ml, qc = eng.mlmc_cfg(M=2, n0_steps=1), eng.qmc_cfg(R=16)
    out = (eng.mcq_types.BookResult * 1)()

    def price(o, ml=ml, qc=qc, mode=0):
        arr = (eng.mcq_types.BookOption * 1)(o)
        return L.mcq_book_price(arr, 1, C.byref(ml), C.byref(qc), mode, out, None)

    assert L.mcq_book_price(None, 1, C.byref(ml), C.byref(qc), 0, out, None) == 1
    assert price(_one(eng), mode=7) == 1
    assert price(_one(eng, d=17)) == 3                                    # wider than 16 assets
    assert b"1..16 assets" in L.mcq_last_error()
    assert price(_one(eng, max_L=12)) == 1
    assert price(_one(eng, max_L=1)) == 1
    assert price(_one(eng, eps=0.0)) == 1
    assert price(_one(eng), qc=eng.qmc_cfg(R=1)) == 3                      # one replica has no variance
    assert price(_one(eng), qc=eng.qmc_cfg(R=33)) == 3
    assert price(_one(eng), ml=eng.mlmc_cfg(M=1, n0_steps=1)) == 1
    assert price(_one(eng, d=16, max_L=11)) == 4                           # 16 x 2^11 dims > 20000
    assert b"20000" in L.mcq_last_error()
    sums = np.zeros((16, 20))
    ps = sums.ctypes.data_as(C.POINTER(C.c_double))
    o = _one(eng)
    assert L.mcq_book_level_sums(C.byref(o), C.byref(ml), C.byref(qc), 5, 0, C.c_int64(64), ps) == 1
    assert L.mcq_book_level_sums(C.byref(o), C.byref(ml), C.byref(qc), 1, C.c_uint32(0xFFFFFF00),
                                 C.c_int64(1024), ps) == 4


def test_config5_book_distributions(eng):
    book = eng.config5_book(n=512, seed=5)
    d = np.array([o.n_assets for o in book])
    assert d.min() == 1 and d.max() == 16
    T = np.array([o.T for o in book])
    eps = np.array([o.eps for o in book])
    L = np.array([o.max_L for o in book])
    assert 0.1 <= T.min() and T.max() <= 3.0
    assert 5e-4 <= eps.min() and eps.max() <= 5e-3
    assert L.min() == 4 and L.max() == 9                                   # 16 .. 512 finest steps
    for o in book[:64]:
        n = o.n_assets
        w = np.ctypeslib.as_array(o.weights, (n,))
        S0 = np.ctypeslib.as_array(o.S0, (n,))
        sig = np.ctypeslib.as_array(o.sigma, (n,))
        Lc = np.ctypeslib.as_array(o.L, (n * n,)).reshape(n, n)
        assert abs(w.sum() - 1) < 1e-12 and (w >= 0).all()
        assert (80 <= S0).all() and (S0 <= 120).all() and (0.1 <= sig).all() and (sig <= 0.5).all()
        corr = Lc @ Lc.T
        assert np.allclose(np.diag(corr), 1.0) and np.allclose(Lc, np.tril(Lc))
        fwd = w @ S0 * np.exp(o.r * o.T)
        assert 0.8 * fwd - 1e-9 <= o.K <= 1.2 * fwd + 1e-9
    # the generator is seeded: the same book twice
    again = eng.config5_book(n=512, seed=5)
    assert all(a.K == b.K and a.n_assets == b.n_assets for a, b in zip(book, again))


def _basket_model(eng, d, seed):
    rng = np.random.default_rng(seed)
    S0 = 100 * rng.uniform(0.8, 1.2, d)
    sig = rng.uniform(0.1, 0.5, d)
    A = rng.normal(size=(d, d))
    Cm = A @ A.T + 0.5 * np.eye(d)
    dg = np.sqrt(np.diag(Cm))
    Lc = np.linalg.cholesky(Cm / np.outer(dg, dg))
    w = rng.dirichlet(np.ones(d))
    return S0, sig, Lc, w


@pytest.mark.parametrize("d,M", [(1, 0), (3, 2), (7, 4)])
def test_oracle_basket_pathwise_delta_is_the_derivative(eng, orc, d, M):
    """Per path, d(Yf - Yc)/dS0_a from the oracle equals a central FP64 difference of Yf - Yc
    (Euler is linear in S0; paths whose basket sits within the bump of K are skipped)."""
    S0, sig, Lc, w = _basket_model(eng, d, 11 + d)
    K, r, T, n_fine = float(w @ S0), 0.03, 1.0, 8
    p = eng.basket(K, r, T, d)
    rng = np.random.default_rng(3)
    h = 1e-5
    checked = 0
    for _ in range(40):
        z = rng.normal(size=n_fine * d)
        m = eng.basket_gbm(S0, sig, L=Lc, weights=w, mu=r, T=T)
        yf, yc, dd = orc.basket_level(m, p, n_fine, M, z)
        for a in range(d):
            up, dn = S0.copy(), S0.copy()
            up[a] += h
            dn[a] -= h
            fu, cu, _ = orc.basket_level(eng.basket_gbm(up, sig, L=Lc, weights=w, mu=r, T=T), p, n_fine, M, z)
            fd, cd, _ = orc.basket_level(eng.basket_gbm(dn, sig, L=Lc, weights=w, mu=r, T=T), p, n_fine, M, z)
            fdiff = ((fu - cu) - (fd - cd)) / (2 * h)
            # skip kinks: payoff piecewise linear in S0, the FD straddles K only within h
            if abs(fu - fd) > 0 and (fu == 0.0) != (fd == 0.0):
                continue
            if M > 0 and (cu == 0.0) != (cd == 0.0):
                continue
            assert abs(fdiff - dd[a]) < 1e-6 * (1 + abs(dd[a])), (a, fdiff, dd[a])
            checked += 1
    assert checked > 20 * d


def test_oracle_basket_level0_matches_the_uncoupled_path(eng, orc):
    """Level 0 of the coupled pair is the plain basket path of orc_path_payoff."""
    S0, sig, Lc, w = _basket_model(eng, 5, 2)
    m = eng.basket_gbm(S0, sig, L=Lc, weights=w, mu=0.03, T=1.5)
    p = eng.basket(float(w @ S0) * 0.95, 0.03, 1.5, 5)
    z = np.random.default_rng(4).normal(size=16 * 5)
    yf, yc, _ = orc.basket_level(m, p, 16, 0, z)
    assert yc == 0.0
    assert abs(yf - orc.path_payoff(m, p, 16, z)) < 1e-12 * (1 + abs(yf))


def test_book_object_copies_and_validates(eng):
    """mcq_book_create / submit / size / clear / free without a GPU: the book copies its options
    (the caller's arrays may go away) and rejects bad ones at submission."""
    b = eng.Book()
    assert len(b) == 0
    opts = [_one(eng, d=d) for d in (1, 5, 16)]
    b.submit(opts)
    del opts
    import gc
    gc.collect()
    assert len(b) == 3
    b.submit([_one(eng, d=2)])
    assert len(b) == 4
    with pytest.raises(eng.MCQError) as e:
        b.submit([_one(eng, d=17)])
    assert e.value.code == 3 and len(b) == 4          # nothing appended on error
    b.clear()
    assert len(b) == 0
    L = eng.lib()
    ml, qc = eng.mlmc_cfg(M=2, n0_steps=1), eng.qmc_cfg(R=16)
    out = (eng.mcq_types.BookResult * 1)()
    assert L.mcq_book_run(b.h, C.byref(ml), C.byref(qc), 0, out, None) == 1   # empty book
    b.close()


@pytest.mark.parametrize("M", [0, 2, 4])
def test_oracle_dupire_basket_own_s0_deltas_vs_fd(eng, orc, M):
    """Dupire basket with each asset's volatility scaled by its own S0 (MCQ_FLAG_BASKET_OWN_S0): the
    path is homogeneous of degree one in (S0_a, S_a), so dd[a] = w_a / S0_a (gf Sf_a - gc Sc_a) is
    the total derivative of the coupled pair dY with respect to S0_a (the scale moving too).  FP64
    central differences path by path; with the reference's asset-0 scale the deltas are 0."""
    d = 4
    S0, _, Lc, _ = _basket_model(eng, d, 7)
    K, r, T, n_fine = float(S0.mean()), 0.03, 1.0, 8
    p = eng.basket(K, r, T, d)
    F = eng.FLAG_BASKET_OWN_S0
    rng = np.random.default_rng(5)
    h = 1e-5
    checked = 0
    for _ in range(30):
        z = rng.normal(size=n_fine * d)
        m = eng.multi_dupire(S0, Lc, mu=r, T=T)
        yf, yc, dd = orc.basket_level(m, p, n_fine, M, z, flags=F)
        _, _, dd0 = orc.basket_level(m, p, n_fine, M, z)
        assert not dd0.any()
        for a in range(d):
            up, dn = S0.copy(), S0.copy()
            up[a] += h
            dn[a] -= h
            fu, cu, _ = orc.basket_level(eng.multi_dupire(up, Lc, mu=r, T=T), p, n_fine, M, z, flags=F)
            fd, cd, _ = orc.basket_level(eng.multi_dupire(dn, Lc, mu=r, T=T), p, n_fine, M, z, flags=F)
            if (fu == 0.0) != (fd == 0.0) or (M > 0 and (cu == 0.0) != (cd == 0.0)):
                continue
            fdiff = ((fu - cu) - (fd - cd)) / (2 * h)
            assert abs(fdiff - dd[a]) < 1e-6 * (1 + abs(dd[a])), (a, fdiff, dd[a])
            checked += 1
    assert checked > 10 * d


def test_oracle_dupire_basket_level0_matches_the_uncoupled_path(eng, orc):
    """Level 0 of the coupled Dupire basket pair is the reference's plain Dupire basket path
    (kernel_multi_dupire, asset 0's S0 in every asset's volatility), and the own-S0 flag reaches
    both."""
    S0, _, Lc, _ = _basket_model(eng, 3, 9)
    m = eng.multi_dupire(S0, Lc, mu=0.03, T=1.5)
    p = eng.basket(float(S0.mean()), 0.03, 1.5, 3)
    z = np.random.default_rng(6).normal(size=16 * 3)
    vals = []
    for flags in (0, eng.FLAG_BASKET_OWN_S0):
        yf, yc, _ = orc.basket_level(m, p, 16, 0, z, flags=flags)
        assert yc == 0.0
        ref = orc.path_payoff(m, p, 16, z, flags=flags)
        assert abs(yf - ref) < 1e-12 * (1 + abs(yf)), (flags, yf, ref)
        vals.append(yf)
    assert vals[0] != vals[1]
