"""Fused pass sums vs the FP64 oracle on the same points, for every model x payoff the
reference supports (plus the down-and-out barrier and the grid local-vol model).

Tolerance: the engine steps paths in FP32 (as the reference) and the oracle in FP64 on the
same normals, so per-replica means agree to ~1e-5 relative; barrier payoffs may flip a
knock-out decision for a path whose extremum sits within FP32 rounding of the barrier, which
moves a mean by at most (max payoff)/N — that bound is added for barrier payoffs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PAYOFFS = ["eur", "asian", "geom", "lookback", "upout", "downout"]


def make_payoff(eng, name, T=1.0):
    return {
        "eur": lambda: eng.european(100.0, 0.05, T),
        "asian": lambda: eng.asian(100.0),
        "geom": lambda: eng.geom_asian(100.0),
        "lookback": lambda: eng.lookback(0.2),
        "upout": lambda: eng.barrier_up_out(100.0, 125.0, 0.2, 0.05, T),
        "downout": lambda: eng.barrier_down_out(100.0, 85.0, 0.2, 0.05, T),
    }[name]()


def make_model(eng, name):
    if name == "gbm":
        return eng.gbm(100.0, 0.05, 0.2, 1.0)
    if name == "heston":
        return eng.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    if name == "dupire":
        return eng.dupire(100.0, 0.05, 0.2, 0.5, 0.7, 1.0)
    if name == "lv":
        K = np.linspace(50, 150, 64)
        t = np.linspace(0, 2, 32)
        g = 0.2 + 0.1 * np.exp(-(K[None, :] / 100 - 1) ** 2 / 0.05) * (1 + 0.5 * t[:, None])
        return eng.localvol_grid(K, t, g, 100.0, 0.05, 1.0)
    raise ValueError(name)


def tol(pay, N, mean):
    t = 2e-4 * (1 + abs(mean))
    if pay in ("upout", "downout"):
        t += 60.0 / N
    return t


@pytest.mark.parametrize("model", ["gbm", "heston", "dupire", "lv"])
@pytest.mark.parametrize("pay", PAYOFFS)
def test_qmc_pass_raw(gpu, orc, model, pay):
    m, p = make_model(gpu, model), make_payoff(gpu, pay)
    n_steps, R, N, off = 24, 2, 640, 13
    g = gpu.qmc_pass(m, p, n_steps, salt_base=42, R=R, offset=off, n_points=N)
    o = orc.qmc_sums(m, p, n_steps, None, salt_base=42, R=R, offset=off, N=N)
    for r in range(R):
        assert abs(g[r, 0] / N - o[r, 0] / N) < tol(pay, N, o[r, 0] / N), (r, g[r], o[r])
        assert abs(g[r, 1] - o[r, 1]) < 1e-3 * (1 + abs(o[r, 1])) + (4000.0 if pay in ("upout", "downout") else 0)


@pytest.mark.parametrize("model", ["gbm", "dupire", "lv"])
@pytest.mark.parametrize("pay", ["eur", "asian", "lookback", "downout"])
@pytest.mark.parametrize("N_steps", [16, 64])
def test_qmc_pass_bridge(gpu, orc, model, pay, N_steps):
    m, p = make_model(gpu, model), make_payoff(gpu, pay)
    bb = gpu.bb_create(N_steps, 1.0)
    R, N = 2, 512
    g = gpu.qmc_pass(m, p, N_steps, noise=gpu.BB, bb=bb, salt_base=77, R=R, offset=64, n_points=N)
    o = orc.qmc_sums(m, p, N_steps, orc.noise(orc.T.BB, N_steps, 1.0), salt_base=77, R=R, offset=64, N=N)
    for r in range(R):
        assert abs(g[r, 0] / N - o[r, 0] / N) < tol(pay, N, o[r, 0] / N), (r, g[r], o[r])
    bb.close()


@pytest.mark.parametrize("model", ["gbm", "heston", "dupire"])
@pytest.mark.parametrize("pay", ["eur", "asian", "lookback", "downout"])
@pytest.mark.parametrize("level", [0, 1, 3])
@pytest.mark.parametrize("M", [2, 4])
def test_level_pass(gpu, orc, model, pay, level, M):
    m, p = make_model(gpu, model), make_payoff(gpu, pay)
    n0 = 1 if M == 2 else 4
    n_fine = n0 * M ** level
    Mp = M if level > 0 else 0
    R, N = 2, 384
    for use_sobol in (True, False):
        g = gpu.level_pass(m, p, n_fine, Mp, use_sobol=use_sobol, seed=42, salt_base=90, R=R, offset=5, n_points=N)
        o = orc.level_sums(m, p, n_fine, Mp, None, use_sobol=use_sobol, seed=42, salt_base=90, R=R, offset=5, N=N)
        for r in range(R):
            for k in (0, 2):
                assert abs(g[r, k] / N - o[r, k] / N) < tol(pay, N, o[r, k] / N) * 2, (use_sobol, r, k, g[r], o[r])


def test_heston_mlmc_compat_flag_skips_running_update(gpu, orc):
    m, p = make_model(gpu, "heston"), make_payoff(gpu, "lookback")
    N = 256
    for flags in (0, gpu.FLAG_COMPAT_HESTON_MLMC):
        g = gpu.level_pass(m, p, 16, 4, use_sobol=True, salt_base=3, R=1, n_points=N, flags=flags)
        o = orc.level_sums(m, p, 16, 4, None, use_sobol=True, salt_base=3, R=1, N=N, flags=flags)
        assert abs(g[0, 2] / N - o[0, 2] / N) < 1e-3, flags


@pytest.mark.parametrize("model,pay", [("gbm", "eur"), ("heston", "asian"), ("dupire", "lookback"), ("lv", "geom")])
def test_mc_pass_philox(gpu, orc, model, pay):
    m, p = make_model(gpu, model), make_payoff(gpu, pay)
    N = 700
    g = gpu.mc_pass(m, p, 40, 123, 5, 1000, N)
    o = orc.mc_sums(m, p, 40, 123, 5, 1000, N)
    assert abs(g[0] / N - o[0] / N) < 2e-4 * (1 + abs(o[0] / N)), (g, o)


@pytest.mark.parametrize("kind", ["multi", "basket"])
@pytest.mark.parametrize("n", [1, 3, 8, 16])
def test_basket_pass(gpu, orc, kind, n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n))
    Cm = A @ A.T + 0.5 * np.eye(n)
    d = np.sqrt(np.diag(Cm))
    L = np.linalg.cholesky(Cm / np.outer(d, d))
    S0 = 100 * rng.uniform(0.8, 1.2, n)
    if kind == "multi":
        m = gpu.multi_dupire(S0, L)
    else:
        m = gpu.basket_gbm(S0, rng.uniform(0.1, 0.5, n), L, rng.dirichlet(np.ones(n)))
    p = gpu.basket(100.0, 0.05, 1.0, n)
    R, N, steps = 2, 256, 12
    g = gpu.qmc_pass(m, p, steps, salt_base=11, R=R, offset=3, n_points=N)
    o = orc.qmc_sums(m, p, steps, None, salt_base=11, R=R, offset=3, N=N)
    for r in range(R):
        assert abs(g[r, 0] / N - o[r, 0] / N) < 3e-4 * (1 + abs(o[r, 0] / N)), (r, g[r], o[r])


def test_cv_pilot_matches_pathwise_oracle(gpu, orc):
    m = gpu.gbm(100.0, 0.05, 0.2, 1.0)
    pa, pg = gpu.asian(100.0), gpu.geom_asian(100.0)
    n_steps, N, seed = 16, 1500, 7
    E = orc.geom_asian(100, 100, 1, 0.05, 0.2, n_steps)
    got = gpu.cv_pilot(m, m, pa, pg, E, n_steps, N, seed)
    ya, yg = [], []
    for i in range(N):
        z = orc.philox_normals(seed, 0, i, n_steps)
        ya.append(orc.path_payoff(m, pa, n_steps, z))
        yg.append(orc.path_payoff(m, pg, n_steps, z))
    ya, yg = np.array(ya), np.array(yg)
    va = ya.var()
    vg = max(1e-30, yg.var())
    cov = (ya * yg).mean() - ya.mean() * yg.mean()
    assert abs(got["var_plain"] - va) < 1e-4 * va
    assert abs(got["beta"] - np.clip(cov / vg, 0, 5)) < 1e-4


@pytest.mark.parametrize("model,pay", [("gbm", "asian"), ("heston", "lookback"), ("dupire", "eur")])
def test_launch_variants_are_bit_identical(gpu, model, pay):
    import os
    m, p = make_model(gpu, model), make_payoff(gpu, pay)
    out = []
    try:
        for v in ("0", "1", "2"):
            os.environ["MCQ_TUNE"] = v
            out.append(gpu.qmc_pass(m, p, 64, salt_base=42, R=4, offset=3, n_points=400000))
    finally:
        os.environ.pop("MCQ_TUNE", None)
    assert gpu.debug_last_pass_layout()[0] >= 2   # items of several groups: carried start words in play
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


@pytest.mark.parametrize("model,pay", [("gbm", "asian"), ("heston", "lookback"), ("dupire", "eur")])
def test_coupled_launch_variants_are_bit_identical(gpu, model, pay):
    """The coupled MLMC / MLQMC level pass under its three launch variants (two register budgets,
    and the unrolled tile generator)."""
    import os
    m, p = make_model(gpu, model), make_payoff(gpu, pay)
    out = []
    try:
        for v in ("0", "1", "2"):
            os.environ["MCQ_TUNE"] = v
            out.append(gpu.level_pass(m, p, 64, 4, use_sobol=True, salt_base=42, R=4, offset=3, n_points=400000))
    finally:
        os.environ.pop("MCQ_TUNE", None)
    assert gpu.debug_last_pass_layout()[0] >= 2
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


@pytest.mark.parametrize("model,pay", [("gbm", "asian"), ("dupire", "eur")])
def test_bridge_launch_variants_are_bit_identical(gpu, model, pay):
    import os
    m, p = make_model(gpu, model), make_payoff(gpu, pay)
    bb = gpu.bb_create(256, m.T)
    out = []
    try:
        for v in ("0", "1", "2"):   # a uniform time grid: the window weights come from the parameters
            os.environ["MCQ_TUNE"] = v
            out.append(gpu.qmc_pass(m, p, 256, noise=gpu.BB, bb=bb, salt_base=42, R=4, offset=3, n_points=320000))
    finally:
        os.environ.pop("MCQ_TUNE", None)
        bb.close()
    assert gpu.debug_last_pass_layout()[0] >= 2
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


@pytest.mark.parametrize("pay", ["eur", "lookback", "downout"])
def test_heston_milstein_flag(gpu, orc, pay):
    """MCQ_FLAG_HESTON_MILSTEIN (Euler-Milstein variance step): single-level and coupled level
    sums against the FP64 oracle with the same flag, and the flag changes the result."""
    m, p = make_model(gpu, "heston"), make_payoff(gpu, pay)
    F, N, R = gpu.FLAG_HESTON_MILSTEIN, 1024, 2
    g = gpu.qmc_pass(m, p, 64, salt_base=42, R=R, offset=0, n_points=N, flags=F)
    o = orc.qmc_sums(m, p, 64, None, salt_base=42, R=R, offset=0, N=N, flags=F)
    e = orc.qmc_sums(m, p, 64, None, salt_base=42, R=R, offset=0, N=N, flags=0)
    for r in range(R):
        assert abs(g[r, 0] / N - o[r, 0] / N) < tol(pay, N, o[r, 0] / N), (r, g[r], o[r])
    assert np.abs(o[:, 1] - e[:, 1]).max() > 1e-9 * np.abs(e[:, 1]).max()   # the term is there
    gl = gpu.level_pass(m, p, 64, 4, use_sobol=True, salt_base=7, R=R, n_points=N, flags=F)
    ol = orc.level_sums(m, p, 64, 4, None, use_sobol=True, salt_base=7, R=R, N=N, flags=F)
    for r in range(R):
        for k in (0, 2):
            assert abs(gl[r, k] / N - ol[r, k] / N) < tol(pay, N, ol[r, k] / N) * 2, (r, k, gl[r], ol[r])



def _top_points(orc, salt, dims, n=1 << 22):
    """First point index per dimension whose scrambled word is >= 0xFFFFFF80 (u rounds to 1)."""
    out = {}
    for dim in dims:
        hit = np.nonzero(orc.sobol_hh_u32(salt, dim, 1, 0, n)[0] >= 0xFFFFFF80)[0]
        if len(hit):
            out[dim] = int(hit[0])
    return out


@pytest.mark.parametrize("parity", [0, 1])
@pytest.mark.parametrize("pay", ["eur", "lookback"])
def test_heston_compat_u_inf_matches_reference(gpu, orc, parity, pay):
    """Under MCQ_FLAG_COMPAT_U_INF a scrambled word >= 0xFFFFFF80 gives u = 1 and an infinite
    normal (methods_cuda.cu:823).  In the reference's Heston step (:276-284) that normal makes
    S or V infinite, a truncated variance then gives 0 * inf = NaN in S, and fmaxf drops the NaN
    in the payoff.  The engine must take the same path to the same sums (oracle = the reference's
    formulas in FP64), for a hit on the first (z1, even dimension) and the second (z2, odd
    dimension) normal of a step, single level and coupled; in particular the Milstein term must
    not turn an infinite variance into NaN when it is off.  The default mode stays finite."""
    m, p = make_model(gpu, "heston"), make_payoff(gpu, pay)
    hits = _top_points(orc, 42, [d for d in range(64) if d % 2 == parity])
    assert hits
    dim, x = min(hits.items(), key=lambda kv: kv[0])
    off, N, C = (x // 32) * 32, 32, gpu.FLAG_COMPAT_U_INF

    def same(a, b):
        fa, fb = np.isfinite(a), np.isfinite(b)
        if fa != fb:
            return False
        return (not fa) or abs(a / N - b / N) < tol(pay, N, b / N)

    g = gpu.qmc_pass(m, p, 32, salt_base=42, R=1, offset=off, n_points=N, flags=C)
    o = orc.qmc_sums(m, p, 32, None, salt_base=42, R=1, offset=off, N=N, flags=C)
    o0 = orc.qmc_sums(m, p, 32, None, salt_base=42, R=1, offset=off, N=N)
    if pay == "lookback":
        assert np.isnan(o[0, 0])                  # the NaN path reaches the lookback payoff
    assert same(g[0, 0], o[0, 0]), (dim, g, o)
    gl = gpu.level_pass(m, p, 32, 4, use_sobol=True, salt_base=42, R=1, offset=off, n_points=N, flags=C)
    ol = orc.level_sums(m, p, 32, 4, None, use_sobol=True, salt_base=42, R=1, offset=off, N=N, flags=C)
    assert same(gl[0, 2], ol[0, 2]) and same(gl[0, 0], ol[0, 0]), (dim, gl, ol)
    g0 = gpu.qmc_pass(m, p, 32, salt_base=42, R=1, offset=off, n_points=N)
    assert np.isfinite(g0[0, 0]) and abs(g0[0, 0] / N - o0[0, 0] / N) < tol(pay, N, o0[0, 0] / N)


@pytest.mark.parametrize("use_sobol", [True, False])
@pytest.mark.parametrize("K,z_star,n_steps", [(100.0, 0.5, 64), (180.0, 3.0, 100), (140.0, 1.5, 37)])
def test_is_pass_vs_oracle(gpu, orc, use_sobol, K, z_star, n_steps):
    """The importance-sampling pass (IsC; kernel_is_gbm, methods_cuda.cu:685-707) path by path in the
    FP64 oracle on the same normals: drift-shifted Euler path, likelihood ratio, weighted payoff.
    Per-replica means and second moments to FP32 rounding."""
    m, p = gpu.gbm(100.0, 0.05, 0.2, 1.0), gpu.european(K, 0.05, 1.0)
    zs = z_star / np.sqrt(n_steps)
    R, N = 3, 2000
    g = gpu.is_pass(m, p, n_steps, zs, use_sobol=use_sobol, seed=9, salt_base=31, R=R, offset=17, n_points=N)
    o = orc.is_sums(m, p, n_steps, zs, use_sobol=use_sobol, seed=9, salt_base=31, R=R, offset=17, N=N)
    for r in range(R):
        assert abs(g[r, 0] / N - o[r, 0] / N) < 2e-4 * (1 + abs(o[r, 0] / N)), (r, g[r], o[r])
        assert abs(g[r, 1] - o[r, 1]) < 1e-3 * (1 + abs(o[r, 1])), (r, g[r], o[r])
    # the shift and the likelihood ratio are applied: the sums differ from those of z* = 0
    g0 = gpu.is_pass(m, p, n_steps, 0.0, use_sobol=use_sobol, seed=9, salt_base=31, R=R, offset=17, n_points=N)
    assert np.abs(g0[:, 0] - g[:, 0]).max() > 1e-3 * np.abs(g[:, 0]).max()


def _corr_basket(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    Cm = A @ A.T + 0.5 * np.eye(n)
    d = np.sqrt(np.diag(Cm))
    return 100 * rng.uniform(0.8, 1.2, n), np.linalg.cholesky(Cm / np.outer(d, d))


@pytest.mark.parametrize("flags", [0, 16])
@pytest.mark.parametrize("n", [1, 3, 8, 16])
@pytest.mark.parametrize("level,M", [(0, 2), (1, 2), (3, 2), (1, 4), (2, 4)])
def test_dupire_basket_level_pass(gpu, orc, n, level, M, flags):
    """The coupled Dupire basket (the reference's kernel_multi_dupire path stepped as kernel_mlmc
    steps a one-asset Dupire path; the reference refuses it at methods_cuda.cu:1318-1320) against the
    FP64 oracle's pair on the same scrambled points, with the reference's asset-0 volatility scale
    and with MCQ_FLAG_BASKET_OWN_S0 (16)."""
    S0, L = _corr_basket(n, 40 + n)
    m = gpu.multi_dupire(S0, L, mu=0.04, T=1.0)
    p = gpu.basket(float(S0.mean()), 0.04, 1.0, n)
    nf = M ** level
    R, N = 2, 512
    g = gpu.level_pass(m, p, nf, M if level else 0, use_sobol=True, salt_base=70, R=R, offset=9, n_points=N,
                       flags=flags)
    o = orc.basket_level_sums(m, p, nf, M if level else 0, salt_base=70, R=R, offset=9, N=N, flags=flags)
    for r in range(R):
        sc = 1 + abs(o[r, 2] / N)
        assert abs(g[r, 0] / N - o[r, 0] / N) < 3e-4 * sc, (r, g[r], o[r, :4])
        assert abs(g[r, 2] / N - o[r, 2] / N) < 3e-4 * sc, (r, g[r], o[r, :4])


def test_dupire_basket_own_s0_single_level(gpu, orc):
    """MCQ_FLAG_BASKET_OWN_S0 in the single-level Dupire basket pass (BasketC and the wide basket):
    against the oracle with the flag, and different from the reference's asset-0 scale."""
    for n in (5, 40):
        S0, L = _corr_basket(n, 3)
        m = gpu.multi_dupire(S0, L, mu=0.04, T=1.0)
        p = gpu.basket(float(S0.mean()), 0.04, 1.0, n)
        R, N, steps = 2, 256, 8
        got = {}
        for flags in (0, gpu.FLAG_BASKET_OWN_S0):
            g = gpu.qmc_pass(m, p, steps, salt_base=21, R=R, offset=0, n_points=N, flags=flags)
            o = orc.qmc_sums(m, p, steps, None, salt_base=21, R=R, offset=0, N=N, flags=flags)
            for r in range(R):
                assert abs(g[r, 0] / N - o[r, 0] / N) < 3e-4 * (1 + abs(o[r, 0] / N)), (n, flags, g[r], o[r])
            got[flags] = g
        assert np.abs(got[0][:, 0] - got[gpu.FLAG_BASKET_OWN_S0][:, 0]).max() > 1e-6 * N


@pytest.mark.parametrize("flags", [0, 16])
def test_dupire_basket_mlmc_mlqmc(gpu, flags):
    """MLMC and MLQMC of a 4-asset Dupire basket (refused by the reference) telescope to the plain
    estimator at their finest level: compared with it within 3 standard
    errors of the difference plus the bias bound eps / sqrt(2) of the stopping test (the plain
    estimator: single-level RQMC at that step count, independent salts)."""
    S0, L = _corr_basket(4, 8)
    m = gpu.multi_dupire(S0, L, mu=0.03, T=1.0)
    p = gpu.basket(float(S0.mean()), 0.03, 1.0, 4)
    eps = 2e-2
    ml = gpu.run_mlmc(m, p, eps, gpu.mlmc_cfg(M=2, max_L=8, flags=flags))
    q = gpu.run_mlqmc(m, p, eps, gpu.mlmc_cfg(M=2, max_L=8, flags=flags), gpu.qmc_cfg(R=16, flags=flags))
    for r in (ml, q):
        finest = 2 ** (r["levels"] - 1)
        ref = gpu.run_qmc(m, p, eps / 2, finest, gpu.qmc_cfg(R=16, N0_per_replica=1 << 12, salt_base=900, flags=flags))
        assert abs(r["price"] - ref["price"]) < 3 * np.hypot(r["std_error"], ref["std_error"]) + eps / np.sqrt(2), (r, ref)


@pytest.mark.parametrize("pay", ["lookback", "downout"])
@pytest.mark.parametrize("level,R,N", [(3, 2, 2048), (5, 2, 1024), (7, 1, 256), (8, 1, 128)])
def test_heston_fine_levels_vs_oracle(gpu, orc, pay, level, R, N):
    """The Heston MLQMC workload's own levels (Euler-Milstein variance, M = 4, 4 steps on level 0;
    level 8 is 262,144 steps) on the same normals as the FP64 oracle: Sobol while the level fits the
    20,000-dimension table, Philox beyond.  At these step sizes FP32 rounding must stay unbiased: a
    rounded e^{-kappa h} near 1, or the drift of a fine step added to S on its own, would shift the
    means systematically (by ~4e-3 on the lookback at level 8)."""
    m = make_model(gpu, "heston")
    p = gpu.lookback(0.2) if pay == "lookback" else gpu.barrier_down_out(100.0, 80.0, 0.2, 0.02, 1.0)
    F = gpu.FLAG_HESTON_MILSTEIN
    nf = 4 * 4 ** level
    sob = nf * 2 <= 20000
    g = gpu.level_pass(m, p, nf, 4, use_sobol=sob, seed=11, salt_base=600, R=R, offset=0, n_points=N, flags=F)
    o = orc.level_sums(m, p, nf, 4, None, use_sobol=sob, seed=11, salt_base=600, R=R, offset=0, N=N, flags=F)
    for r in range(R):
        sc = 1 + abs(o[r, 2] / N)
        extra = 60.0 / N if pay == "downout" else 0.0
        assert abs(g[r, 2] / N - o[r, 2] / N) < 2e-4 * sc + extra, (level, r, g[r], o[r])
        assert abs(g[r, 0] / N - o[r, 0] / N) < 2e-4 * sc + extra, (level, r, g[r], o[r])


def test_bench_pass_at_full_size_vs_fp64_oracle(gpu):
    """The benchmark's own pass (arithmetic Asian, 256 steps, 32 replicas x 2^20 scrambled-Sobol
    points) against the FP64 oracle's per-replica sums on the same points, replica by replica
    (tests/golden/oracle_values.json, written by make_oracle_values.py): FP32 paths, FP64 sums."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "oracle_values.json")) as f:
        ref = json.load(f)["asian_gbm_256_engine_points"]
    R, N = ref["R"], ref["N"]
    o = np.array(ref["sums"])
    g = gpu.qmc_pass(gpu.gbm(100.0, 0.03, 0.25, 1.0), gpu.asian(100.0), 256, salt_base=ref["salt_base"], R=R,
                     offset=0, n_points=N)
    gm, om = g[:, 0] / N, o[:, 0] / N
    assert np.abs(gm - om).max() < 2e-5 * (1 + np.abs(om).max()), np.abs(gm - om).max()
    assert abs(gm.mean() - om.mean()) < 5e-6 * om.mean()
