"""Assisted passes: raw-ordered passes with few 32-path groups and long paths, where three helper
warps generate each path-owning warp's normals.  On one B200 (148 SMs) a pass is assisted when it
has fewer than 148 x 8 groups and at least 256 normals per path.  The same points priced as
replica 0 of a one-replica pass (assisted, 800 groups) and of a two-replica pass (1600 groups, the
plain loop) have the same work items, so their sums must agree bit for bit; the oracle checks the
values."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_ASSIST = 800 * 32   # 800 groups: assisted with one replica, not with two


def _model(gpu, name):
    if name == "gbm":
        return gpu.gbm(100.0, 0.05, 0.2, 1.0)
    if name == "heston":
        return gpu.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    if name == "dupire":
        return gpu.dupire(100.0, 0.05, 0.2, 0.5, 0.7, 1.0)
    K = np.linspace(50, 150, 64)
    t = np.linspace(0, 2, 32)
    g = 0.2 + 0.1 * np.exp(-(K[None, :] / 100 - 1) ** 2 / 0.05) * (1 + 0.5 * t[:, None])
    return gpu.localvol_grid(K, t, g, 100.0, 0.05, 1.0)


def _payoff(gpu, name):
    return {"eur": lambda: gpu.european(100.0, 0.05, 1.0), "asian": lambda: gpu.asian(100.0),
            "lookback": lambda: gpu.lookback(0.2),
            "downout": lambda: gpu.barrier_down_out(100.0, 85.0, 0.2, 0.05, 1.0)}[name]()


@pytest.mark.parametrize("model,steps", [("gbm", 300), ("heston", 128), ("dupire", 260), ("lv", 256)])
@pytest.mark.parametrize("pay", ["asian", "lookback"])
def test_assisted_pass_equals_plain_loop(gpu, model, steps, pay):
    m, p = _model(gpu, model), _payoff(gpu, pay)
    one = gpu.qmc_pass(m, p, steps, salt_base=42, R=1, offset=5, n_points=N_ASSIST)
    two = gpu.qmc_pass(m, p, steps, salt_base=42, R=2, offset=5, n_points=N_ASSIST)
    assert np.array_equal(one[0], two[0]), (one, two)


@pytest.mark.parametrize("model", ["gbm", "heston", "dupire"])
@pytest.mark.parametrize("use_sobol", [True, False])
def test_assisted_coupled_level_equals_plain_loop(gpu, model, use_sobol):
    m, p = _model(gpu, model), _payoff(gpu, "lookback")
    kw = dict(use_sobol=use_sobol, seed=42, salt_base=90, offset=3, n_points=N_ASSIST)
    one = gpu.level_pass(m, p, 256, 4, R=1, **kw)
    two = gpu.level_pass(m, p, 256, 4, R=2, **kw)
    assert np.array_equal(one[0], two[0]), (one, two)


@pytest.mark.parametrize("model,steps", [("gbm", 256), ("heston", 130), ("dupire", 270), ("lv", 288)])
@pytest.mark.parametrize("pay", ["eur", "asian", "downout"])
def test_assisted_pass_vs_oracle(gpu, orc, model, steps, pay):
    m, p = _model(gpu, model), _payoff(gpu, pay)
    R, N, off = 2, 1500, 11
    g = gpu.qmc_pass(m, p, steps, salt_base=7, R=R, offset=off, n_points=N)
    o = orc.qmc_sums(m, p, steps, None, salt_base=7, R=R, offset=off, N=N)
    for r in range(R):
        t = 2e-4 * (1 + abs(o[r, 0] / N)) + (60.0 / N if pay == "downout" else 0.0)
        assert abs(g[r, 0] / N - o[r, 0] / N) < t, (r, g[r], o[r])


@pytest.mark.parametrize("use_sobol", [True, False])
def test_assisted_coupled_level_vs_oracle(gpu, orc, use_sobol):
    m, p = _model(gpu, "heston"), _payoff(gpu, "lookback")
    R, N = 2, 1000
    g = gpu.level_pass(m, p, 256, 4, use_sobol=use_sobol, seed=42, salt_base=90, R=R, offset=3, n_points=N)
    o = orc.level_sums(m, p, 256, 4, None, use_sobol=use_sobol, seed=42, salt_base=90, R=R, offset=3, N=N)
    for r in range(R):
        for k in (0, 2):
            assert abs(g[r, k] / N - o[r, k] / N) < 2e-4 * (1 + abs(o[r, k] / N)), (r, k, g[r], o[r])
