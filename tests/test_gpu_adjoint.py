"""Pathwise adjoint Greeks (mcq_adjoint) against closed forms, against FP64 central finite
differences of the oracle on the same scrambled-Sobol points (h = 1e-4), per grid node of the
local-vol surface, and through a torch.autograd.Function (test harness only)."""
import numpy as np
import pytest
from scipy.stats import norm

pytestmark = pytest.mark.gpu


def oracle_price(orc, m, p, n_steps, salt, R, N):
    s = orc.qmc_sums(m, p, n_steps, None, salt, R, 0, N)
    return s[:, 0].sum() / (R * N)


def fd(orc, build, p, n_steps, x0, salt=7, R=1, N=4096, rel=1e-4):
    h = rel * max(abs(x0), 1e-2)
    up = oracle_price(orc, build(x0 + h), p, n_steps, salt, R, N)
    dn = oracle_price(orc, build(x0 - h), p, n_steps, salt, R, N)
    return (up - dn) / (2 * h)


def test_gbm_european_matches_black_scholes(gpu):
    S0, K, r, s, T = 100.0, 100.0, 0.05, 0.2, 1.0
    g, _ = gpu.adjoint(gpu.gbm(S0, r, s, T), gpu.european(K, r, T), 256, R=16, n_points=1 << 16)
    d1 = (np.log(S0 / K) + (r + 0.5 * s * s) * T) / (s * np.sqrt(T))
    d2 = d1 - s * np.sqrt(T)
    bs = {"price": S0 * norm.cdf(d1) - K * np.exp(-r * T) * norm.cdf(d2), "delta": norm.cdf(d1),
          "vega": S0 * norm.pdf(d1) * np.sqrt(T), "rho": K * T * np.exp(-r * T) * norm.cdf(d2)}
    for k, v in bs.items():
        assert abs(g[k] - v) < 4 * g[k + "_se"] + 5e-3 * abs(v), (k, g[k], v, g[k + "_se"])


@pytest.mark.parametrize("pay", ["asian", "eur", "lookback"])
def test_gbm_greeks_vs_fp64_finite_differences(gpu, orc, pay):
    T = orc.T
    S0, mu, s, n = 100.0, 0.03, 0.25, 64
    mk = {"asian": lambda: T.asian(100.0), "eur": lambda: T.european(100.0, mu, 1.0), "lookback": lambda: T.lookback(0.25)}
    p = mk[pay]()
    g, _ = gpu.adjoint(gpu.gbm(S0, mu, s, 1.0), p, n, salt_base=7, R=1, n_points=4096)
    delta = fd(orc, lambda x: T.gbm(x, mu, s, 1.0), p, n, S0)
    vega = fd(orc, lambda x: T.gbm(S0, mu, x, 1.0), p, n, s)
    if pay == "eur":   # drift and discount move together
        rho = fd(orc, lambda x: T.gbm(S0, x, s, 1.0), T.european(100.0, mu, 1.0), n, mu)
        rho += (oracle_price(orc, T.gbm(S0, mu, s, 1.0), T.european(100.0, mu + 1e-6, 1.0), n, 7, 1, 4096) -
                oracle_price(orc, T.gbm(S0, mu, s, 1.0), T.european(100.0, mu - 1e-6, 1.0), n, 7, 1, 4096)) / 2e-6
    else:
        rho = fd(orc, lambda x: T.gbm(S0, x, s, 1.0), p, n, mu)
    for name, ref in (("delta", delta), ("vega", vega), ("rho", rho)):
        assert abs(g[name] - ref) < 2e-4 * max(1.0, abs(ref)), (pay, name, g[name], ref)


def test_local_vol_node_vegas_vs_fp64_finite_differences(gpu, orc):
    T = orc.T
    K, t, grid = gpu.config4_surface()
    n, N = 64, 4096
    m = gpu.localvol_grid(K, t, grid, 100.0, 0.05, 2.0)
    p = T.asian(100.0)
    g, nodes = gpu.adjoint(m, p, n, salt_base=11, R=1, n_points=N)
    assert nodes.shape == (32, 64)
    assert abs(nodes.sum() - g["vega"]) < 1e-6 * max(1, abs(g["vega"]))
    # the eight most sensitive nodes, bumped one at a time in the FP64 oracle
    order = np.argsort(-np.abs(nodes).ravel())[:8]
    for idx in order:
        j, i = divmod(int(idx), 64)

        def build(x, j=j, i=i):
            g2 = grid.copy()
            g2[j, i] = x
            return T.localvol_grid(K, t, g2, 100.0, 0.05, 2.0)

        ref = fd(orc, build, p, n, grid[j, i], salt=11, N=N)
        if abs(nodes[j, i] - ref) < 1e-3 * abs(ref) + 2e-5:
            continue
        # The price is piecewise smooth in a node (the bilinear surface has kinks in S at the strike
        # nodes, and near t = 0 many paths sit close to one): when a kink falls inside the bump the
        # central difference at h = 1e-4 is biased.  Then the adjoint must lie in the bracket of the
        # one-sided differences and match the central difference with the kink resolved (h = 1e-6).
        # The payoff kink of one path whose average lies within FP32 rounding of the strike may
        # fall on different sides in the FP32 adjoint and the FP64 oracle; that path alone moves
        # the node sensitivity by its pathwise weight / N (about 0.5% here at N = 4096), so the
        # bracket and the fine difference are held to 1%.
        h = 1e-4 * grid[j, i]
        v0 = oracle_price(orc, build(grid[j, i]), p, n, 11, 1, N)
        up = (oracle_price(orc, build(grid[j, i] + h), p, n, 11, 1, N) - v0) / h
        dn = (v0 - oracle_price(orc, build(grid[j, i] - h), p, n, 11, 1, N)) / h
        assert min(up, dn) - 1e-2 * abs(ref) <= nodes[j, i] <= max(up, dn) + 1e-2 * abs(ref), (j, i, nodes[j, i], up, dn)
        fine = fd(orc, build, p, n, grid[j, i], salt=11, N=N, rel=1e-6)
        assert abs(nodes[j, i] - fine) < 1e-2 * abs(fine) + 2e-5, (j, i, nodes[j, i], fine)
    # delta: the bilinear surface's strike kinks are crossed by thousands of path-steps within a
    # bump of 1e-4 S0, which biases that central difference by ~1e-3; at 1e-7 S0 the FP64
    # difference has converged (it agrees with 1e-8 S0 to 2e-7)
    dl = fd(orc, lambda x: T.localvol_grid(K, t, grid, x, 0.05, 2.0), p, n, 100.0, salt=11, N=N, rel=1e-7)
    assert abs(g["delta"] - dl) < 2e-4, (g["delta"], dl)


def test_config4_full_size_runs(gpu):
    K, t, grid = gpu.config4_surface()
    m = gpu.localvol_grid(K, t, grid, 100.0, 0.05, 2.0)
    g, nodes = gpu.adjoint(m, gpu.asian(100.0), 512, salt_base=42, R=16, n_points=1 << 18)
    assert g["n_paths"] == 16 * (1 << 18) and np.isfinite(nodes).all()
    assert 0 < g["delta"] < 1 and g["vega"] > 0 and g["price_se"] < 0.05


def test_torch_autograd_wrapper(gpu):
    import torch

    class McqPrice(torch.autograd.Function):
        """Price of a GBM Asian call as a differentiable function of (S0, sigma, mu); the
        backward pass is the engine's pathwise adjoint."""

        @staticmethod
        def forward(ctx, S0, sigma, mu):
            g, _ = gpu.adjoint(gpu.gbm(float(S0), float(mu), float(sigma), 1.0), gpu.asian(100.0), 64,
                               salt_base=3, R=4, n_points=4096)
            ctx.save_for_backward(torch.tensor([g["delta"], g["vega"], g["rho"]], dtype=torch.float64))
            return torch.tensor(g["price"], dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad):
            (gr,) = ctx.saved_tensors
            return grad * gr[0], grad * gr[1], grad * gr[2]

    S0 = torch.tensor(100.0, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(0.25, dtype=torch.float64, requires_grad=True)
    mu = torch.tensor(0.03, dtype=torch.float64, requires_grad=True)
    price = McqPrice.apply(S0, sig, mu)
    dS, dsig, dmu = torch.autograd.grad(price, [S0, sig, mu])
    h = 1e-3
    m = lambda s0, sg, u: McqPrice.apply(torch.tensor(s0), torch.tensor(sg), torch.tensor(u)).item()
    assert abs(dS.item() - (m(100 + h, 0.25, 0.03) - m(100 - h, 0.25, 0.03)) / (2 * h)) < 1e-3
    assert abs(dsig.item() - (m(100, 0.25 + 1e-4, 0.03) - m(100, 0.25 - 1e-4, 0.03)) / 2e-4) < 2e-2


def _heston_price(orc, m, p, n, salt, N, flags):
    s = orc.qmc_sums(m, p, n, None, salt, 1, 0, N, flags)
    return s[0, 0] / N


@pytest.mark.parametrize("pay,flags", [("eur", 0), ("asian", 0), ("lookback", 0), ("asian", 8)])
def test_heston_adjoint_vs_fp64_finite_differences(gpu, orc, pay, flags):
    """Heston (full truncation; flags 8 adds the Milstein variance term): pathwise delta, rho and
    dP/dv0 against FP64 central differences of the oracle on the same scrambled points."""
    T = orc.T
    S0, mu, kap, th, xi, rho_c, v0 = 100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04
    n, N = 64, 4096

    def model(S0=S0, mu=mu, v0=v0):
        return T.heston(S0, mu, kap, th, xi, rho_c, v0, 1.0)

    p = {"eur": T.european(100.0, mu, 1.0), "asian": T.asian(100.0), "lookback": T.lookback(0.2)}[pay]
    g, _ = gpu.adjoint(model(), p, n, salt_base=7, R=1, n_points=N, flags=flags)

    def fd(build, x0, rel=1e-4):
        hh = rel * x0
        return (_heston_price(orc, build(x0 + hh), p, n, 7, N, flags) -
                _heston_price(orc, build(x0 - hh), p, n, 7, N, flags)) / (2 * hh)

    delta = fd(lambda x: model(S0=x), S0)
    vega = fd(lambda x: model(v0=x), v0)
    if pay == "eur":   # the drift and the discount share the rate
        rho = fd(lambda x: model(mu=x), mu)
        pu, pd = T.european(100.0, mu + 1e-6, 1.0), T.european(100.0, mu - 1e-6, 1.0)
        rho += (orc.qmc_sums(model(), pu, n, None, 7, 1, 0, N, flags)[0, 0] -
                orc.qmc_sums(model(), pd, n, None, 7, 1, 0, N, flags)[0, 0]) / N / 2e-6
    else:
        rho = fd(lambda x: model(mu=x), mu)
    price = _heston_price(orc, model(), p, n, 7, N, flags)
    assert abs(g["price"] - price) < 2e-4 * max(1.0, abs(price)), (g["price"], price)
    for name, ref in (("delta", delta), ("rho", rho), ("vega", vega)):
        assert abs(g[name] - ref) < 2e-3 * max(1.0, abs(ref)), (pay, name, g[name], ref)


@pytest.mark.parametrize("model,pay", [("gbm", "asian"), ("heston", "eur"), ("heston", "asian"), ("gbm", "lookback"),
                                       ("dupire", "asian"), ("dupire", "lookback")])
def test_adjoint_delta_vs_bump_and_revalue_through_the_pricer(gpu, model, pay):
    """Pathwise delta against bump-and-revalue of the pricing pass itself (the restated reference
    pricer, FP32, common scrambled points, bump 1% of S0).  Not the grid surface: its strike kinks
    bias any central difference at a bump the FP32 pricer can resolve (it is checked against
    converged FP64 differences above)."""
    if model == "gbm":
        build = lambda s: gpu.gbm(s, 0.05, 0.2, 1.0)
    elif model == "heston":
        build = lambda s: gpu.heston(s, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    else:
        build = lambda s: gpu.dupire(s, 0.05, 0.2, 0.5, 0.7, 1.0)
    p = {"asian": gpu.asian(100.0), "eur": gpu.european(100.0, 0.02, 1.0), "lookback": gpu.lookback(0.2)}[pay]
    n, N, R = 64, 1 << 15, 4
    g, _ = gpu.adjoint(build(100.0), p, n, salt_base=5, R=R, n_points=N)
    up = gpu.qmc_pass(build(101.0), p, n, salt_base=5, R=R, n_points=N)[:, 0].sum() / (R * N)
    dn = gpu.qmc_pass(build(99.0), p, n, salt_base=5, R=R, n_points=N)[:, 0].sum() / (R * N)
    bump = (up - dn) / 2.0
    assert abs(g["delta"] - bump) < 5e-3 * max(1.0, abs(bump)), (model, pay, g["delta"], bump)


@pytest.mark.parametrize("pay", ["eur", "asian", "lookback"])
def test_dupire_adjoint_vs_fp64_finite_differences(gpu, orc, pay):
    """Parametric Dupire: delta (with respect to the model's S0, which also scales the local
    volatility), vega = dP/dsigma0 and rho against FP64 central differences of the oracle."""
    T = orc.T
    mu, s0, al, be = 0.05, 0.2, 0.5, 0.7
    n, N = 64, 4096
    p = {"eur": T.european(100.0, mu, 1.0), "asian": T.asian(100.0), "lookback": T.lookback(0.2)}[pay]
    g, _ = gpu.adjoint(gpu.dupire(100.0, mu, s0, al, be, 1.0), p, n, salt_base=7, R=1, n_points=N)
    delta = fd(orc, lambda x: T.dupire(x, mu, s0, al, be, 1.0), p, n, 100.0)
    vega = fd(orc, lambda x: T.dupire(100.0, mu, x, al, be, 1.0), p, n, s0)
    rho = fd(orc, lambda x: T.dupire(100.0, x, s0, al, be, 1.0), p, n, mu)
    if pay == "eur":
        rho += (oracle_price(orc, T.dupire(100.0, mu, s0, al, be, 1.0), T.european(100.0, mu + 1e-6, 1.0), n, 7, 1, N) -
                oracle_price(orc, T.dupire(100.0, mu, s0, al, be, 1.0), T.european(100.0, mu - 1e-6, 1.0), n, 7, 1, N)) / 2e-6
    for name, ref in (("delta", delta), ("vega", vega), ("rho", rho)):
        assert abs(g[name] - ref) < 5e-4 * max(1.0, abs(ref)), (pay, name, g[name], ref)


@pytest.mark.parametrize("model,pay", [("gbm", "asian"), ("dupire", "eur"), ("lv", "asian"), ("gbm", "lookback")])
def test_checkpoint_interval_variants_are_bit_identical(gpu, model, pay):
    """The adjoint's checkpoint interval (16, 32 or 8 steps: the autotuner's launch variants) only
    changes how many steps a reverse segment recomputes: price, delta, rho and vega are the same
    bits under every variant, the node vegas the same up to the order of their FP32 atomics."""
    import os
    m = {"gbm": lambda: gpu.gbm(100.0, 0.03, 0.25, 1.0), "dupire": lambda: gpu.dupire(100.0, 0.05, 0.2, 0.5, 0.7, 1.0),
         "lv": lambda: gpu.localvol_grid(*gpu.config4_surface(), 100.0, 0.05, 2.0)}[model]()
    p = {"asian": gpu.asian(100.0), "eur": gpu.european(100.0, 0.05, 1.0), "lookback": gpu.lookback(0.25)}[pay]
    out = []
    try:
        for v in ("0", "1", "2"):
            os.environ["MCQ_TUNE"] = v
            out.append(gpu.adjoint(m, p, 128, salt_base=42, R=4, n_points=8192))
    finally:
        os.environ.pop("MCQ_TUNE", None)
    for g, nodes in out[1:]:
        for k in ("price", "delta", "rho", "vega"):
            assert g[k] == out[0][0][k], (k, g[k], out[0][0][k])
        if nodes is not None and out[0][1] is not None:
            # FP32 atomics: only the order of the adds differs
            assert np.abs(nodes - out[0][1]).max() < 1e-5 * np.abs(out[0][1]).max()
