"""Short raw-ordered Sobol paths (at most 16 normals: the low MLMC / MLQMC levels and few-step
passes), which the engine runs with 32 / D path groups per Sobol tile, against the oracle on the
same points; ragged ranges and splits that cut through a tile's groups."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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


def _close(g, o, N, pay):
    t = 2e-4 * (1 + abs(o / N)) + (60.0 / N if pay == "downout" else 0.0)
    return abs(g / N - o / N) < t


@pytest.mark.parametrize("model,steps", [("gbm", 1), ("gbm", 2), ("gbm", 3), ("gbm", 5), ("gbm", 13), ("gbm", 16),
                                         ("heston", 1), ("heston", 3), ("heston", 8),
                                         ("dupire", 4), ("dupire", 11), ("lv", 7), ("lv", 16)])
@pytest.mark.parametrize("pay", ["eur", "asian", "lookback", "downout"])
def test_packed_pass_vs_oracle(gpu, orc, model, steps, pay):
    m, p = _model(gpu, model), _payoff(gpu, pay)
    R, N, off = 2, 3333, 13
    g = gpu.qmc_pass(m, p, steps, salt_base=42, R=R, offset=off, n_points=N)
    o = orc.qmc_sums(m, p, steps, None, salt_base=42, R=R, offset=off, N=N)
    for r in range(R):
        assert _close(g[r, 0], o[r, 0], N, pay), (r, g[r], o[r])


@pytest.mark.parametrize("model,n0,M", [("gbm", 1, 2), ("gbm", 1, 4), ("heston", 1, 2), ("heston", 4, 4),
                                        ("dupire", 1, 2)])
@pytest.mark.parametrize("pay", ["eur", "lookback"])
def test_packed_coupled_levels_vs_oracle(gpu, orc, model, n0, M, pay):
    """The coupled fine / coarse pair on every level whose fine path has at most 16 normals."""
    m, p = _model(gpu, model), _payoff(gpu, pay)
    d = 2 if model == "heston" else 1
    R, N = 2, 2000
    level = 0
    while n0 * M ** level * d <= 16:
        nf = n0 * M ** level
        Mp = M if level > 0 else 0
        g = gpu.level_pass(m, p, nf, Mp, use_sobol=True, salt_base=90, R=R, offset=7, n_points=N)
        o = orc.level_sums(m, p, nf, Mp, None, use_sobol=True, salt_base=90, R=R, offset=7, N=N)
        for r in range(R):
            for k in (0, 2):
                assert _close(g[r, k], o[r, k], N, pay), (level, r, k, g[r], o[r])
        level += 1
    assert level >= 1


@pytest.mark.parametrize("steps", [1, 3, 16])
def test_packed_ragged_splits_add_up(gpu, steps):
    """Ranges cut at points that split a tile's groups: every path is counted once.  One path is
    about 1e-5 of the total here; the tolerance covers the FP32 compensated per-lane sums."""
    m, p = gpu.gbm(100.0, 0.05, 0.2, 1.0), gpu.asian(100.0)
    whole = gpu.qmc_pass(m, p, steps, salt_base=5, R=3, offset=9, n_points=100003)
    parts = sum(gpu.qmc_pass(m, p, steps, salt_base=5, R=3, offset=a, n_points=b - a)
                for a, b in [(9, 40), (40, 41), (41, 1000), (1000, 60001), (60001, 100012)])
    np.testing.assert_allclose(parts, whole, rtol=2e-6)


def test_packed_mlqmc_converges_to_black_scholes(gpu, orc):
    """The MLQMC driver in the reference's level-0-of-one-step form, whose low levels are all
    packed passes."""
    m, p = gpu.gbm(100.0, 0.05, 0.2, 1.0), gpu.european(100.0, 0.05, 1.0)
    q = gpu.run_mlqmc(m, p, 2e-3, gpu.mlmc_cfg(M=2, n0_steps=1, max_L=10), gpu.qmc_cfg(R=16))
    bs = orc.bs_call(100, 100, 1, 0.05, 0.2)
    assert abs(q["price"] - bs) < 4 * q["std_error"] + 2e-3 / np.sqrt(2), q
