"""Adaptive drivers end to end through the C ABI, each result stated against an FP64 oracle
(closed forms where they exist)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_mc_european_vs_black_scholes(gpu, orc):
    m, p = gpu.gbm(100, 0.05, 0.2, 1.0), gpu.european(100, 0.05, 1.0)
    r = gpu.run_mc(m, p, 1e-2, 64, gpu.mc_cfg(pilot_n=1 << 14))
    bs = orc.bs_call(100, 100, 1, 0.05, 0.2)
    assert r["std_error"] < 1e-2
    assert abs(r["price"] - bs) < 4 * r["std_error"] + 0.01, r


def test_mc_fixed_matches_mc_pass(gpu):
    m, p = gpu.gbm(), gpu.asian(100.0)
    mean, var = gpu.run_mc_fixed(m, p, 32, 5000, 99)
    s = gpu.mc_pass(m, p, 32, 99, 0, 0, 5000)
    assert mean == s[0] / 5000
    assert abs(var - max(0.0, s[1] / 5000 - mean ** 2) / 5000) < 1e-15


def test_qmc_asian_raw_and_bridge_agree(gpu, orc):
    m, p = gpu.gbm(100, 0.03, 0.25, 1.0), gpu.asian(100.0)
    cfg = gpu.qmc_cfg(R=32, N0_per_replica=1 << 12)
    raw = gpu.run_qmc(m, p, 2e-3, 256, cfg)
    bb = gpu.bb_create(256, 1.0)
    br = gpu.run_qmc(m, p, 2e-3, 256, cfg, noise=gpu.BB, bb=bb)
    bb.close()
    assert raw["std_error"] < 2e-3 and br["std_error"] < 2e-3
    assert abs(raw["price"] - br["price"]) < 4 * np.hypot(raw["std_error"], br["std_error"]), (raw, br)
    o = orc.run_qmc(m, p, 1.0, 256, None, R=8, max_doublings=1, N0=1 << 11)   # FP64 oracle, fixed size
    assert abs(raw["price"] - o["price"]) < 4 * np.hypot(raw["std_error"], o["std_error"])


def test_qmc_is_deterministic(gpu):
    m, p = gpu.gbm(100, 0.03, 0.25, 1.0), gpu.asian(100.0)
    cfg = gpu.qmc_cfg(R=8, N0_per_replica=1 << 10, max_doublings=1)
    a = gpu.run_qmc(m, p, 1e-9, 128, cfg)
    b = gpu.run_qmc(m, p, 1e-9, 128, cfg)
    assert a["price"] == b["price"] and a["std_error"] == b["std_error"]


def test_mlmc_and_mlqmc_european(gpu, orc):
    m, p = gpu.gbm(100, 0.05, 0.2, 1.0), gpu.european(100, 0.05, 1.0)
    bs = orc.bs_call(100, 100, 1, 0.05, 0.2)
    r = gpu.run_mlmc(m, p, 1e-2)
    assert abs(r["price"] - bs) < 4 * r["std_error"] + 1e-2 / np.sqrt(2), r
    q = gpu.run_mlqmc(m, p, 5e-3, gpu.mlmc_cfg(), gpu.qmc_cfg(R=16))
    assert abs(q["price"] - bs) < 4 * q["std_error"] + 5e-3 / np.sqrt(2), q


def test_mlqmc_bridge_levels(gpu, orc):
    m, p = gpu.gbm(100, 0.05, 0.2, 1.0), gpu.european(100, 0.05, 1.0)
    bbs = [gpu.bb_create(1 << l, 1.0) for l in range(11)]
    q = gpu.run_mlqmc(m, p, 5e-3, gpu.mlmc_cfg(), gpu.qmc_cfg(R=16), noise=gpu.BB, bb_list=bbs)
    bs = orc.bs_call(100, 100, 1, 0.05, 0.2)
    assert abs(q["price"] - bs) < 4 * q["std_error"] + 5e-3 / np.sqrt(2), q
    for b in bbs:
        b.close()


def test_heston_mlmc_config3_shapes(gpu):
    # MLMC telescopes to its finest level, so compare with plain MC at that step count: the
    # lookback's level means decay slowly (BGK-corrected discrete minimum), so MC at a coarser
    # grid differs by the remaining level terms (about 0.13 between 256 and 16384 steps).
    m = gpu.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    ml = gpu.mlmc_cfg(M=4, max_L=8, n0_steps=4)
    look = gpu.run_mlmc(m, gpu.lookback(0.2), 1e-2, ml)
    finest = 4 * 4 ** (look["levels"] - 1)
    mc_look = gpu.run_mc(m, gpu.lookback(0.2), 2e-2, finest)
    assert abs(look["price"] - mc_look["price"]) < 4 * np.hypot(look["std_error"], mc_look["std_error"]), (look, mc_look)
    dno = gpu.run_mlmc(m, gpu.barrier_down_out(100.0, 80.0, 0.2, 0.02, 1.0), 1e-2, ml)
    finest = 4 * 4 ** (dno["levels"] - 1)
    mc_dno = gpu.run_mc(m, gpu.barrier_down_out(100.0, 80.0, 0.2, 0.02, 1.0), 2e-2, finest)
    assert abs(dno["price"] - mc_dno["price"]) < 4 * np.hypot(dno["std_error"], mc_dno["std_error"]), (dno, mc_dno)


def test_control_variate_and_importance_sampling(gpu, orc):
    m = gpu.gbm(100, 0.05, 0.2, 1.0)
    n = 64
    E = orc.geom_asian(100, 100, 1, 0.05, 0.2, n)
    pil = gpu.cv_pilot(m, m, gpu.asian(100.0), gpu.geom_asian(100.0), E, n, 50000)
    assert 0.5 < pil["beta"] < 1.5 and pil["var_cv"] < 0.05 * pil["var_plain"]
    cv = gpu.run_mc_cv(m, m, gpu.asian(100.0), gpu.geom_asian(100.0), E, pil["beta"], 5e-3, n)
    qcv = gpu.run_qmc_cv(m, m, gpu.asian(100.0), gpu.geom_asian(100.0), E, pil["beta"], 5e-3, n,
                         gpu.qmc_cfg(N0_per_replica=1 << 10))
    assert abs(cv["price"] - qcv["price"]) < 4 * np.hypot(cv["std_error"], qcv["std_error"]) + 1e-3
    p180 = gpu.european(180.0, 0.05, 1.0)
    zs = (np.log(1.8) - (0.05 - 0.02)) / 0.2
    r = gpu.run_is(m, p180, zs, 2e-3)
    assert abs(r["price"] - orc.bs_call(100, 180, 1, 0.05, 0.2)) < 4 * r["std_error"] + 2e-3, r


def test_dupire_cv(gpu, orc):
    m = gpu.dupire(100, 0.05, 0.2, 0.5, 0.7, 1.0)
    p = gpu.european(100.0, 0.05, 1.0)
    E = orc.bs_call(100, 100, 1, 0.05, 0.2)
    pil = gpu.cv_pilot(m, gpu.gbm(), p, p, E, 64, 50000)
    assert 0 < pil["beta"] <= 5 and pil["var_cv"] < pil["var_plain"]


def test_range_errors(gpu):
    m, p = gpu.gbm(), gpu.asian(100.0)
    with pytest.raises(gpu.MCQError) as e:
        gpu.run_qmc(m, p, 1e-12, 64, gpu.qmc_cfg(R=2, N0_per_replica=1 << 33, max_doublings=3))
    assert e.value.code == 4
    with pytest.raises(gpu.MCQError) as e:
        gpu.qmc_pass(m, p, 20001, n_points=32)
    assert e.value.code == 4


def _mlmc_restated(gpu, m, p, eps, M, max_L, pilot_n, n0, seed=42):
    """run_mlmc_cuda's adaptive loop (methods_cuda.cu:1305-1487) in Python over the engine's
    level passes, with the engine driver's stream assignment (one fresh stream per launch)."""
    ctr = [0]
    E, V, N = [0.0] * (max_L + 1), [0.0] * (max_L + 1), [0] * (max_L + 1)

    def run(l, n):
        s = gpu.level_pass(m, p, n0 * M ** l, M if l else 0, use_sobol=False, seed=seed, salt_base=ctr[0], R=1,
                           offset=0, n_points=n)[0]
        ctr[0] += 1
        return s

    L = 2
    for l in range(L + 1):
        s = run(l, pilot_n)
        E[l] = s[0] / pilot_n
        V[l] = max(0.0, s[1] / pilot_n - E[l] ** 2)
        N[l] = pilot_n
    conv, it = False, 0
    while not conv and L <= max_L and it < 50:
        it += 1
        st = sum(np.sqrt(V[l] * float(M) ** l) for l in range(L + 1))
        extra = [0] * (L + 1)
        for l in range(L + 1):
            nopt = max(int(np.ceil(2.0 / eps ** 2 * np.sqrt(V[l] / float(M) ** l) * st)), 100)
            if nopt > N[l]:
                extra[l] = nopt - N[l]
        for l in range(L + 1):
            if extra[l]:
                s = run(l, extra[l])
                nn = N[l] + extra[l]
                ts = E[l] * N[l] + s[0]
                t2 = (V[l] + E[l] ** 2) * N[l] + s[1]
                E[l] = ts / nn
                V[l] = max(0.0, t2 / nn - E[l] ** 2)
                N[l] = nn
        b = abs(E[L]) / (M - 1)
        if L >= 1:
            b = max(b, abs(E[L - 1]) * M / (M * M - M))
        conv = b < eps / np.sqrt(2)
        if not conv and L < max_L:
            L += 1
            s = run(L, pilot_n)
            E[L] = s[0] / pilot_n
            V[L] = max(0.0, s[1] / pilot_n - E[L] ** 2)
            N[L] = pilot_n
    return sum(E[:L + 1]), np.sqrt(sum(V[l] / N[l] for l in range(L + 1))), E[:L + 1], N[:L + 1]


@pytest.mark.parametrize("case", ["gbm_eur", "heston_lookback"])
def test_mlmc_driver_equals_restatement(gpu, case):
    if case == "gbm_eur":
        m, p, M, n0, eps = gpu.gbm(100, 0.05, 0.2, 1.0), gpu.european(100, 0.05, 1.0), 2, 1, 2e-2
    else:
        m, p, M, n0, eps = gpu.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0), gpu.lookback(0.2), 4, 4, 2e-2
    r = gpu.run_mlmc(m, p, eps, gpu.mlmc_cfg(M=M, max_L=8, n0_steps=n0))
    price, se, E, N = _mlmc_restated(gpu, m, p, eps, M, 8, 400, n0)
    print(case, r, price, se, E, N)
    assert abs(r["price"] - price) < 1e-12 * max(1, abs(price)), (r, price, E, N)
    assert abs(r["std_error"] - se) < 1e-9
