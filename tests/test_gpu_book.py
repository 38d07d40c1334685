"""Batched heterogeneous book through the C ABI: the book kernel's slice sums against the FP64
oracle, batched == plain bit for bit, agreement with the single-option MLQMC driver, and
prices / deltas against Black–Scholes for one-asset baskets."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ncdf(x):
    return 0.5 * math.erfc(-x / math.sqrt(2.0))


def _basket(eng, d, seed, eps=2e-3, max_L=5, T=1.0, r=0.03, corr=True, kmul=1.0):
    rng = np.random.default_rng(seed)
    S0 = 100 * rng.uniform(0.8, 1.2, d)
    sig = rng.uniform(0.1, 0.5, d)
    A = rng.normal(size=(d, d))
    Cm = A @ A.T + 0.5 * np.eye(d)
    dg = np.sqrt(np.diag(Cm))
    Lc = np.linalg.cholesky(Cm / np.outer(dg, dg)) if corr else None
    w = rng.dirichlet(np.ones(d))
    K = float(kmul * (w @ S0) * np.exp(r * T))
    o = eng.book_option(S0, sig, K, r, T, eps, max_L, weights=w, L=Lc)
    return o, (S0, sig, Lc, w, K, r, T)


@pytest.mark.parametrize("d,level,corr", [(1, 0, True), (3, 1, True), (4, 3, False), (7, 2, True),
                                          (12, 1, True), (16, 4, True),
                                          # long step-major paths; paired tiles at d = 11, 12
                                          (7, 5, True), (9, 4, True), (11, 3, False), (12, 5, True)])
def test_book_slice_sums_match_oracle(gpu, orc, d, level, corr):
    """Per-replica sums of one slice (ragged offset and count) through the book kernel against
    the FP64 oracle of the coupled basket pair with pathwise deltas."""
    o, (S0, sig, Lc, w, K, r, T) = _basket(gpu, d, 100 + d, corr=corr)
    ml, qc = gpu.mlmc_cfg(M=2, n0_steps=1), gpu.qmc_cfg(R=4, salt_base=42)
    offset, N = 37, 1000
    g = gpu.book_level_sums(o, level, offset, N, ml, qc)
    m = gpu.basket_gbm(S0, sig, L=Lc, weights=w, mu=r, T=T)
    p = gpu.basket(K, r, T, d)
    ref = orc.basket_level_sums(m, p, 2 ** level, 2 if level else 0, salt_base=42 + level * 4, R=4,
                                offset=offset, N=N)
    # FP32 paths against FP64: 2e-5 of the per-point scale of the payoff (columns 0, 2) and
    # of its square (columns 1, 3), summed over the N points
    for q in range(4):
        scale = N + abs(ref[:, 3 if q in (1, 3) else 2]).max()
        assert np.abs(g[:, q] - ref[:, q]).max() < 2e-5 * scale, (q, g[:, q], ref[:, q])
    # deltas: a path whose basket sits within FP32 rounding of K may flip its indicator
    assert np.abs(g[:, 4:] - ref[:, 4:]).max() < 3.0 + 1e-4 * N, (g[:, 4:], ref[:, 4:])


def test_book_batched_equals_plain_bit_for_bit(gpu):
    book = gpu.config5_book(n=24, seed=77)
    for o in book:
        o.eps = 10 * o.eps                       # keep the test short: coarser targets
    rb, sb = gpu.book_price(book, gpu.BOOK_BATCHED)
    rp, sp = gpu.book_price(book, gpu.BOOK_PLAIN)
    for a, b in zip(rb, rp):
        assert a["price"] == b["price"] and a["std_error"] == b["std_error"]
        assert a["n_samples"] == b["n_samples"] and a["levels"] == b["levels"]
        assert np.array_equal(a["delta"], b["delta"])
    assert sb["path_steps"] == sp["path_steps"]
    assert sb["launches"] < sp["launches"]


def test_book_matches_single_option_mlqmc(gpu):
    """Each option of a book against run_mlqmc on the same basket: the same points and MLQMC
    logic, but the slice sums are reduced in a different order, and an FP64 rounding difference
    can tip a ceil() in the sample-size rule, after which the two runs draw different points.
    So: prices within 3 combined standard errors, finest levels within one."""
    opts, models = [], []
    for i, d in enumerate([1, 2, 5, 9, 16]):
        o, (S0, sig, Lc, w, K, r, T) = _basket(gpu, d, 300 + i, eps=3e-3, max_L=6, T=0.5 + 0.4 * i)
        opts.append(o)
        models.append((gpu.basket_gbm(S0, sig, L=Lc, weights=w, mu=r, T=T), gpu.basket(K, r, T, d)))
    res, _ = gpu.book_price(opts, gpu.BOOK_BATCHED, gpu.mlmc_cfg(M=2, n0_steps=1), gpu.qmc_cfg(R=16))
    for o, (m, p), b in zip(opts, models, res):
        ml = gpu.mlmc_cfg(M=2, n0_steps=1, max_L=o.max_L)
        ref = gpu.run_mlqmc(m, p, o.eps, ml, gpu.qmc_cfg(R=16))
        assert abs(b["levels"] - ref["levels"]) <= 1, (b, ref)
        assert abs(b["price"] - ref["price"]) < 3 * np.hypot(b["std_error"], ref["std_error"]), (b, ref)
        assert 0.5 < b["std_error"] / ref["std_error"] < 2.0, (b, ref)


@pytest.mark.parametrize("seed,kmul,T", [(9, 1.0, 1.0), (10, 0.9, 0.5), (10, 1.0, 1.0)])
def test_book_one_asset_vs_black_scholes(gpu, orc, seed, kmul, T):
    """A one-asset basket is a European call: once the MLQMC bias test has passed, the price is
    within 3 SE + 10 eps of Black–Scholes (the stopping rule |E_L| / (M - 1) < eps / sqrt 2 of
    run_mlqmc_cuda bounds the Euler bias only heuristically) and the pathwise delta within 1e-2
    of N(d1).  Volatilities near 0.2, so that the bias test passes by level 10."""
    o, (S0, sig, _, w, K, r, T) = _basket(gpu, 1, seed, eps=1e-3, max_L=10, T=T, kmul=kmul)
    (res,), _ = gpu.book_price([o], gpu.BOOK_BATCHED)
    assert res["converged"], res
    S, s = float(S0[0]), float(sig[0])
    bs = orc.bs_call(S, K, T, r, s)
    d1 = (math.log(S / K) + (r + 0.5 * s * s) * T) / (s * math.sqrt(T))
    assert abs(res["price"] - bs) < 3 * res["std_error"] + 10 * o.eps, (res, bs)
    assert abs(res["delta"][0] - _ncdf(d1)) < 1e-2, (res["delta"], _ncdf(d1))


def test_book_delta_matches_bump_and_revalue(gpu):
    """Pathwise deltas of a 6-asset slice against central differences of the same slice with
    common scrambled points (bump 0.5% of S0)."""
    o, (S0, sig, Lc, w, K, r, T) = _basket(gpu, 6, 900)
    ml, qc = gpu.mlmc_cfg(M=2, n0_steps=4), gpu.qmc_cfg(R=8)
    N = 1 << 14
    g = gpu.book_level_sums(o, 0, 0, N, ml, qc)
    for a in range(6):
        h = 5e-3 * S0[a]
        up, dn = S0.copy(), S0.copy()
        up[a] += h
        dn[a] -= h
        ou = gpu.book_option(up, sig, K, r, T, o.eps, o.max_L, weights=w, L=Lc)
        od = gpu.book_option(dn, sig, K, r, T, o.eps, o.max_L, weights=w, L=Lc)
        fu = gpu.book_level_sums(ou, 0, 0, N, ml, qc)[:, 2].sum()
        fd = gpu.book_level_sums(od, 0, 0, N, ml, qc)[:, 2].sum()
        fdiff = (fu - fd) / (2 * h)
        pw = g[:, 4 + a].sum()
        assert abs(fdiff - pw) < 1e-2 * abs(pw) + 1e-3 * N * w[a], (a, fdiff, pw)


def test_book_config5_sample_prices_converge(gpu):
    """A sample of the synthetic book: every option either passes the bias test or has grown
    to its finest level, every option's SE meets its own eps (converged or not), and the one-asset
    options that converged agree with Black–Scholes within the stopping test's bias bound
    eps / sqrt(2) plus 3 standard errors."""
    book = gpu.config5_book(n=64, seed=5)
    for o in book:
        o.eps = 4 * o.eps                        # keep the test short: coarser targets
    res, st = gpu.book_price(book, gpu.BOOK_BATCHED)
    assert st["rounds"] >= 2 and st["launches"] == 6 * st["rounds"]   # 5 class kernels + finalize
    for o, r in zip(book, res):
        assert np.isfinite(r["price"]) and r["price"] >= 0
        assert r["std_error"] <= o.eps * 1.01, (o.eps, r)
        if o.n_assets == 1 and r["converged"]:
            S, s = o.S0[0], o.sigma[0]
            assert abs(r["price"] - orc_bs(S, o.K, o.T, o.r, s)) < 3 * r["std_error"] + o.eps / math.sqrt(2)
        assert r["converged"] or r["levels"] == o.max_L + 1, (o.max_L, r)


def orc_bs(S, K, T, r, s):
    d1 = (math.log(S / K) + (r + 0.5 * s * s) * T) / (s * math.sqrt(T))
    return S * _ncdf(d1) - K * math.exp(-r * T) * _ncdf(d1 - s * math.sqrt(T))


def _mlqmc_restated(gpu, o, pilot=400, R=16, M=2, n0=1, iter_cap=50):
    """run_mlqmc_cuda's adaptive loop (methods_cuda.cu:1950-2016) restated in Python for one
    option of a book, with every slice priced through the book kernel's per-replica sums."""
    ml, qc = gpu.mlmc_cfg(M=M, n0_steps=n0), gpu.qmc_cfg(R=R)
    nl = o.max_L + 1
    E, sig2, N, off = [0.0] * nl, [0.0] * nl, [0] * nl, [0] * nl
    D = [[0.0] * o.n_assets for _ in range(nl)]

    def run(l, n):
        s = gpu.book_level_sums(o, l, off[l], n, ml, qc)
        stats = []
        for col in [0] + [4 + a for a in range(o.n_assets)]:
            rep = [float(s[r, col]) / n for r in range(R)]
            m = 0.0
            for v in rep:
                m += v
            stats.append((m / R, rep))
        m, rep = stats[0]
        var = 0.0
        for v in rep:
            var += (v - m) * (v - m)
        var = var / (R - 1)
        if N[l] == 0:
            E[l], sig2[l] = m, var * n
            D[l] = [x for x, _ in stats[1:]]
        else:
            wo, wn = float(N[l]), float(n)
            E[l] = (E[l] * wo + m * wn) / (wo + wn)
            sig2[l] = (sig2[l] * wo + var * wn * wn) / (wo + wn)
            D[l] = [(D[l][a] * wo + stats[1 + a][0] * wn) / (wo + wn) for a in range(o.n_assets)]
        N[l] += n
        off[l] += n

    L = 2
    for l in range(3):
        run(l, pilot)
    converged, it = False, 0
    while not converged and L <= o.max_L and it < iter_cap:
        it += 1
        st = 0.0
        for l in range(L + 1):
            st += math.sqrt(sig2[l] * float(M ** l))
        extra = []
        for l in range(L + 1):
            Nopt = max(math.ceil(2.0 / (R * o.eps * o.eps) * math.sqrt(sig2[l] / float(M ** l)) * st), 100)
            if Nopt > N[l]:
                extra.append((l, Nopt - N[l]))
        for l, n in extra:
            run(l, n)
        bias = abs(E[L]) / max(M - 1, 1)
        if L >= 1:
            bias = max(bias, abs(E[L - 1]) * M / max(M * (M - 1), 1))
        converged = bias < o.eps / math.sqrt(2.0)
        if not converged and L < o.max_L:
            L += 1
            run(L, pilot)
    price, vs, Nt = 0.0, 0.0, 0
    delta = [0.0] * o.n_assets
    for l in range(L + 1):
        price += E[l]
        vs += sig2[l] / (float(N[l]) * R)
        Nt += N[l] * R
        for a in range(o.n_assets):
            delta[a] += D[l][a]
    return {"price": price, "std_error": math.sqrt(vs), "n_samples": Nt, "levels": L + 1,
            "converged": converged, "delta": np.array(delta)}


def test_book_state_machine_matches_python_restatement(gpu):
    """The book's per-option MLQMC state machine (rounds of pending slices) against a plain
    restatement of run_mlqmc_cuda's loop driven through the same kernel: same levels, sample
    counts and bits."""
    book = gpu.config5_book(n=6, seed=91)
    for o in book:
        o.eps = 8 * o.eps
        o.max_L = min(o.max_L, 6)
    res, _ = gpu.book_price(book, gpu.BOOK_BATCHED)
    for o, b in zip(book, res):
        ref = _mlqmc_restated(gpu, o)
        assert (b["levels"], b["n_samples"], b["converged"]) == (ref["levels"], ref["n_samples"], ref["converged"])
        assert b["price"] == ref["price"] and b["std_error"] == ref["std_error"], (b, ref)
        assert np.array_equal(b["delta"], ref["delta"])


def test_book_object_run_equals_book_price(gpu):
    """The submit / run book object prices exactly as mcq_book_price on the same options."""
    opts = gpu.config5_book(n=10, seed=33)
    for o in opts:
        o.eps = 10 * o.eps
    ref, _ = gpu.book_price(opts, gpu.BOOK_BATCHED)
    b = gpu.Book()
    b.submit(opts[:4])
    b.submit(opts[4:])
    out, st = b.run(gpu.BOOK_BATCHED)
    b.close()
    for r, o, x in zip(ref, opts, out):
        assert r["price"] == x.price and r["std_error"] == x.std_error and r["n_samples"] == x.n_samples
        assert np.array_equal(r["delta"], np.array(x.delta[:o.n_assets]))


def test_book_class_variants_are_bit_identical(gpu):
    """The book's width classes under both register-budget variants (the autotuner's choices) give
    the same prices, deltas and sample counts, batched and plain."""
    import os
    book = gpu.config5_book(n=4096, seed=5)
    opts = []
    for d in (2, 6, 10, 14):
        o = next(o for o in book if o.n_assets == d)
        c = type(o).from_buffer_copy(o)
        c.eps = 10 * o.eps
        opts.append(c)
    res = []
    try:
        for v in ("0", "1"):
            os.environ["MCQ_TUNE"] = v
            for mode in (gpu.BOOK_BATCHED, gpu.BOOK_PLAIN):
                res.append(gpu.book_price(opts, mode)[0])
    finally:
        os.environ.pop("MCQ_TUNE", None)
    for r in res[1:]:
        for a, b in zip(res[0], r):
            assert a["price"] == b["price"] and a["n_samples"] == b["n_samples"]
            assert np.array_equal(a["delta"], b["delta"])


def _single(gpu, model, pay, eps=5e-3, max_L=6):
    m = {"gbm": lambda: gpu.gbm(100.0, 0.02, 0.25, 1.0),
         "heston": lambda: gpu.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0),
         "dupire": lambda: gpu.dupire(100.0, 0.02, 0.2, 0.5, 0.7, 1.0)}[model]()
    p = {"eur": lambda: gpu.european(100.0, 0.02, 1.0), "asian": lambda: gpu.asian(100.0),
         "lookback": lambda: gpu.lookback(0.2), "downout": lambda: gpu.barrier_down_out(100.0, 85.0, 0.2, 0.02, 1.0),
         "upout": lambda: gpu.barrier_up_out(100.0, 130.0, 0.2, 0.02, 1.0), "geom": lambda: gpu.geom_asian(100.0)}[pay]()
    return gpu.book_single(m, p, eps, max_L), m, p


@pytest.mark.parametrize("model,pay,level", [("gbm", "eur", 0), ("gbm", "asian", 3), ("heston", "lookback", 2),
                                             ("heston", "downout", 4), ("dupire", "eur", 1), ("dupire", "upout", 5),
                                             ("gbm", "geom", 2)])
def test_book_single_asset_slice_sums_match_oracle(gpu, orc, model, pay, level):
    """A single-asset book option's slice through the book's single-asset class kernel (the fused
    pass's coupled consumer) against the FP64 oracle's coupled level pair on the same points
    (salts salt_base + level R + r, a ragged offset and count)."""
    o, m, p = _single(gpu, model, pay)
    ml, qc = gpu.mlmc_cfg(M=2, n0_steps=1), gpu.qmc_cfg(R=4, salt_base=42)
    offset, N = 37, 1000
    g = gpu.book_level_sums(o, level, offset, N, ml, qc)
    ref = orc.level_sums(m, p, 2 ** level, 2 if level else 0, None, use_sobol=True, salt_base=42 + level * 4, R=4,
                         offset=offset, N=N)
    extra = 60.0 if pay in ("downout", "upout") else 0.0
    for q in (0, 2):
        scale = N + abs(ref[:, 2]).max()
        assert np.abs(g[:, q] - ref[:, q]).max() < 2e-5 * scale + extra, (q, g[:, q], ref[:, q])


@pytest.mark.parametrize("model,pay", [("gbm", "eur"), ("heston", "lookback"), ("dupire", "asian")])
def test_book_single_asset_agrees_with_run_mlqmc(gpu, model, pay):
    """A single-asset option priced in the book and by mcq_run_mlqmc: the same model, payoff, levels,
    salts and point counts, so the same paths; the level sums are reduced in different orders, so
    the prices agree to the rounding of the sums unless a rounding tips a sample count, and always
    within 3 standard errors of the difference."""
    o, m, p = _single(gpu, model, pay, eps=3e-3, max_L=6)
    ml, qc = gpu.mlmc_cfg(M=2, n0_steps=1, max_L=6), gpu.qmc_cfg(R=16)
    rb, _ = gpu.book_price([o], gpu.BOOK_BATCHED, ml, qc)
    q = gpu.run_mlqmc(m, p, 3e-3, ml, qc)
    assert abs(rb[0]["price"] - q["price"]) < 3 * np.hypot(rb[0]["std_error"], q["std_error"]), (rb[0], q)
    assert rb[0]["levels"] == q["levels"]
    assert not rb[0]["delta"].any()


def test_mixed_book_batched_equals_plain_and_black_scholes(gpu):
    """Baskets and single-asset options in one book: batched equals plain bit for bit, and the GBM
    European singles that converged lie within the stopping test's bias bound plus 3 standard errors
    of Black-Scholes."""
    book = gpu.config5_book(n=8, seed=77) + gpu.mixed_singles(n=12, seed=3)
    for o in book:
        o.eps = 5 * o.eps
    rb, _ = gpu.book_price(book, gpu.BOOK_BATCHED)
    rp, _ = gpu.book_price(book, gpu.BOOK_PLAIN)
    for a, b in zip(rb, rp):
        assert a["price"] == b["price"] and a["n_samples"] == b["n_samples"]
        assert np.array_equal(a["delta"], b["delta"])
    checked = 0
    for o, r in zip(book, rb):
        if o.model and o.model.contents.kind == gpu.GBM and o.payoff.contents.kind == gpu.EUROPEAN and r["converged"]:
            m, p = o.model.contents, o.payoff.contents
            d1 = (math.log(m.S0 / p.K) + (m.mu + 0.5 * m.sigma ** 2) * m.T) / (m.sigma * math.sqrt(m.T))
            bs = m.S0 * _ncdf(d1) - p.K * math.exp(-p.r * p.T) * _ncdf(d1 - m.sigma * math.sqrt(m.T))
            assert abs(r["price"] - bs) < o.eps / math.sqrt(2) + 3 * r["std_error"], (r, bs)
            checked += 1
    assert checked >= 1


@pytest.mark.parametrize("d,level", [(3, 3), (12, 3), (16, 6)])
def test_book_slice_carried_start_words(gpu, orc, d, level):
    """A slice long enough for chunks of several 32-path groups, where the book kernel carries each
    tile's Sobol start word from group to group (a path's first 24 tiles; the d = 16 path at level 6
    has 32, its last 8 walk theirs; d = 12 generates tile pairs): sums against the FP64 oracle."""
    o, (S0, sig, Lc, w, K, r, T) = _basket(gpu, d, 300 + d, max_L=8)
    ml, qc = gpu.mlmc_cfg(M=2, n0_steps=1), gpu.qmc_cfg(R=4, salt_base=42)
    offset, N = 37, 20000
    g = gpu.book_level_sums(o, level, offset, N, ml, qc)
    m = gpu.basket_gbm(S0, sig, L=Lc, weights=w, mu=r, T=T)
    p = gpu.basket(K, r, T, d)
    ref = orc.basket_level_sums(m, p, 2 ** level, 2, salt_base=42 + level * 4, R=4, offset=offset, N=N)
    for q in range(4):
        scale = N + abs(ref[:, 3 if q in (1, 3) else 2]).max()
        assert np.abs(g[:, q] - ref[:, q]).max() < 2e-5 * scale, (q, g[:, q], ref[:, q])


@pytest.mark.parametrize("level", [4, 8, 9])
def test_book_single_asset_carried_start_words(gpu, orc, level):
    """Single-asset chunks of several groups carry their start words when the path has at most 16
    tiles (Heston at level 8: 256 steps x 2 factors = 16 tiles) and walk them beyond (level 9):
    slice sums against the FP64 oracle either way."""
    o, m, p = _single(gpu, "heston", "lookback", max_L=10)
    ml, qc = gpu.mlmc_cfg(M=2, n0_steps=1), gpu.qmc_cfg(R=4, salt_base=42)
    offset, N = 37, 20000
    g = gpu.book_level_sums(o, level, offset, N, ml, qc)
    ref = orc.level_sums(m, p, 2 ** level, 2, None, use_sobol=True, salt_base=42 + level * 4, R=4,
                         offset=offset, N=N)
    for q in (0, 2):
        scale = N + abs(ref[:, 2]).max()
        assert np.abs(g[:, q] - ref[:, q]).max() < 2e-5 * scale, (q, g[:, q], ref[:, q])
