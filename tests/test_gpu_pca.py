"""PCA ordering on the GPU: the tensor-core pass (tcgen05, N in {64, 128, 256}) and the
single-tile pass (N <= 32) against an FP64 product on the same fp16-rounded inputs, the oracle,
and the reference's own cuBLAS PCA pass (tests/golden)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def f16(x):
    return np.asarray(x, np.float32).astype(np.float16).astype(np.float64)


@pytest.mark.parametrize("N", [4, 32, 64, 128, 256])
def test_pca_increments_match_fp64_product(gpu, N):
    pca = gpu.pca_create(N, 1.0)
    M = f16(gpu.pca_matrix(pca))                       # M[i, k] as the device sees it
    R, n, off = 2, 300, 77
    dump = gpu.debug_pass_dump(gpu.gbm(), N, gpu.PCA, bb=pca, use_sobol=True, salt_base=9, R=R, offset=off,
                               n_points=n)
    for r in range(R):
        z = f16(gpu.sobol_hh_normal(9 + r, 0, N, off, n))   # [N, n]
        ref = (M @ z).T                                      # [n, N]
        assert np.allclose(dump[r], ref, atol=2e-6, rtol=2e-5), (r, np.abs(dump[r] - ref).max())
    pca.close()


@pytest.mark.parametrize("N", [32, 64, 256])
@pytest.mark.parametrize("pay", ["asian", "eur", "lookback"])
def test_pca_pass_vs_oracle(gpu, orc, N, pay):
    m = gpu.gbm(100.0, 0.03, 0.25, 1.0)
    p = {"asian": gpu.asian(100.0), "eur": gpu.european(100.0, 0.03, 1.0), "lookback": gpu.lookback(0.25)}[pay]
    pca = gpu.pca_create(N, 1.0)
    R, Np = 2, 2048
    g = gpu.qmc_pass(m, p, N, noise=gpu.PCA, pca=pca, salt_base=42, R=R, offset=0, n_points=Np)
    o = orc.qmc_sums(m, p, N, orc.noise(orc.T.PCA, N, 1.0), salt_base=42, R=R, offset=0, N=Np)
    for r in range(R):
        assert abs(g[r, 0] / Np - o[r, 0] / Np) < 3e-4 * (1 + abs(o[r, 0] / Np)), (r, g[r], o[r])
    pca.close()


def test_pca_pass_equals_reference_cublas_pass(gpu):
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import golden_cases
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_golden.npz"))
    case = {c[0]: c for c in golden_cases.cases(gpu.mcq_types)}["asian_pca_256"]
    _, m, p, n_steps, mode, salt0, R, off, N = case
    pca = gpu.pca_create(n_steps, 1.0)
    mine = gpu.qmc_pass(m, p, n_steps, noise=gpu.PCA, pca=pca, salt_base=salt0, R=R, offset=off, n_points=N)
    ref = gold["pass_asian_pca_256"]
    for r in range(R):
        assert abs(mine[r, 0] / N - ref[r, 0] / N) < 1e-4 * (1 + abs(ref[r, 0] / N)), (r, mine[r], ref[r])
    pca.close()


def test_pca_qmc_driver_and_mlqmc(gpu, orc):
    m, p = gpu.gbm(100.0, 0.03, 0.25, 1.0), gpu.asian(100.0)
    pca = gpu.pca_create(256, 1.0)
    r = gpu.run_qmc(m, p, 2e-3, 256, gpu.qmc_cfg(R=32, N0_per_replica=1 << 12), noise=gpu.PCA, pca=pca)
    raw = gpu.run_qmc(m, p, 2e-3, 256, gpu.qmc_cfg(R=32, N0_per_replica=1 << 12))
    assert abs(r["price"] - raw["price"]) < 4 * np.hypot(r["std_error"], raw["std_error"]), (r, raw)
    pca.close()
    me, pe = gpu.gbm(100, 0.05, 0.2, 1.0), gpu.european(100, 0.05, 1.0)
    lst = [gpu.pca_create(1 << l, 1.0) for l in range(9)]
    q = gpu.run_mlqmc(me, pe, 5e-3, gpu.mlmc_cfg(max_L=8), gpu.qmc_cfg(R=16), noise=gpu.PCA, pca_list=lst)
    bs = orc.bs_call(100, 100, 1, 0.05, 0.2)
    assert abs(q["price"] - bs) < 4 * q["std_error"] + 5e-3 / np.sqrt(2), q
    for h in lst:
        h.close()


def _lv_model(gpu, name):
    if name == "dupire":
        return gpu.dupire(100.0, 0.05, 0.2, 0.5, 0.7, 1.0)
    K = np.linspace(50, 150, 64)
    t = np.linspace(0, 2, 32)
    g = 0.2 + 0.1 * np.exp(-(K[None, :] / 100 - 1) ** 2 / 0.05) * (1 + 0.5 * t[:, None])
    return gpu.localvol_grid(K, t, g, 100.0, 0.05, 1.0)


@pytest.mark.parametrize("model", ["dupire", "lv"])
@pytest.mark.parametrize("N", [64, 128])
def test_pca_pass_local_vol_models_vs_oracle(gpu, orc, model, N):
    """The tensor-core pass with the parametric and the grid local-volatility models."""
    m, p = _lv_model(gpu, model), gpu.asian(100.0)
    pca = gpu.pca_create(N, 1.0)
    R, Np, off = 2, 1500, 21
    g = gpu.qmc_pass(m, p, N, noise=gpu.PCA, pca=pca, salt_base=17, R=R, offset=off, n_points=Np)
    o = orc.qmc_sums(m, p, N, orc.noise(orc.T.PCA, N, 1.0), salt_base=17, R=R, offset=off, N=Np)
    for r in range(R):
        assert abs(g[r, 0] / Np - o[r, 0] / Np) < 3e-4 * (1 + abs(o[r, 0] / Np)), (r, g[r], o[r])
    pca.close()


@pytest.mark.parametrize("model", ["gbm", "dupire"])
@pytest.mark.parametrize("n_fine,M", [(64, 2), (128, 4), (256, 2)])
def test_pca_coupled_level_vs_oracle(gpu, orc, model, n_fine, M):
    """A coupled MLQMC level (fine path on the tensor-core PCA increments, coarse path on their
    M-step sums) against the oracle's level sums."""
    m = _lv_model(gpu, "dupire") if model == "dupire" else gpu.gbm(100.0, 0.05, 0.2, 1.0)
    p = gpu.european(100.0, 0.05, 1.0)
    pca = gpu.pca_create(n_fine, 1.0)
    R, Np = 2, 1024
    g = gpu.level_pass(m, p, n_fine, M, noise=gpu.PCA, pca=pca, use_sobol=True, salt_base=90, R=R, offset=3,
                       n_points=Np)
    o = orc.level_sums(m, p, n_fine, M, orc.noise(orc.T.PCA, n_fine, 1.0), use_sobol=True, salt_base=90, R=R,
                       offset=3, N=Np)
    for r in range(R):
        for k in (0, 2):
            assert abs(g[r, k] / Np - o[r, k] / Np) < 4e-4 * (1 + abs(o[r, k] / Np)), (r, k, g[r], o[r])
    pca.close()


def test_pca_ragged_ranges_add_up(gpu):
    """A range split at points that are not multiples of the 128-path tile gives the sums of the
    whole range: every path is counted once whatever the tiles, work items and TMEM accumulator
    turns.  The tolerance covers the FP32 compensated per-lane sums (one path is 1e-5 of the
    total here)."""
    m, p = gpu.gbm(100.0, 0.03, 0.25, 1.0), gpu.asian(100.0)
    pca = gpu.pca_create(128, 1.0)
    kw = dict(noise=gpu.PCA, pca=pca, salt_base=42, R=3)
    whole = gpu.qmc_pass(m, p, 128, offset=5, n_points=100001, **kw)
    parts = sum(gpu.qmc_pass(m, p, 128, offset=a, n_points=b - a, **kw)
                for a, b in [(5, 133), (133, 134), (134, 50001), (50001, 100006)])
    np.testing.assert_allclose(parts, whole, rtol=2e-6)
    pca.close()


@pytest.mark.parametrize("N", [48, 100, 512, 1024])
@pytest.mark.parametrize("pay", ["asian", "eur"])
def test_pca_large_n_pass_vs_oracle(gpu, orc, N, pay):
    """PCA orderings outside the tensor-core pass's sizes (fp16 normals, the library GEMM of the
    reference's phase1_pca, the fused pass on the increments) against the FP64 oracle's product of
    the same fp16-rounded factor and normals."""
    m = gpu.gbm(100.0, 0.03, 0.25, 1.0)
    p = gpu.asian(100.0) if pay == "asian" else gpu.european(100.0, 0.03, 1.0)
    pca = gpu.pca_create(N, 1.0)
    R, Np = 2, 1024 if N <= 512 else 256
    g = gpu.qmc_pass(m, p, N, noise=gpu.PCA, pca=pca, salt_base=42, R=R, offset=5, n_points=Np)
    o = orc.qmc_sums(m, p, N, orc.noise(orc.T.PCA, N, 1.0), salt_base=42, R=R, offset=5, N=Np)
    for r in range(R):
        assert abs(g[r, 0] / Np - o[r, 0] / Np) < 3e-4 * (1 + abs(o[r, 0] / Np)), (r, g[r], o[r])
    pca.close()


def test_pca_large_n_batches_and_levels(gpu):
    """A 2048-step PCA pass larger than one batch (2^27 / N points) equals the sum of its two halves
    priced separately (only the FP64 summation order differs), and a coupled MLQMC level at 512
    steps runs through the same route."""
    m, p = gpu.gbm(100.0, 0.03, 0.25, 1.0), gpu.asian(100.0)
    N = 2048
    pca = gpu.pca_create(N, 1.0)
    n1 = (1 << 27) // N
    whole = gpu.qmc_pass(m, p, N, noise=gpu.PCA, pca=pca, salt_base=3, R=1, offset=0, n_points=n1 + 1000)
    a = gpu.qmc_pass(m, p, N, noise=gpu.PCA, pca=pca, salt_base=3, R=1, offset=0, n_points=n1)
    b = gpu.qmc_pass(m, p, N, noise=gpu.PCA, pca=pca, salt_base=3, R=1, offset=n1, n_points=1000)
    assert np.allclose(whole, a + b, rtol=1e-12, atol=0), (whole, a + b)
    pca.close()
    pl = gpu.pca_create(512, 1.0)
    lv = gpu.level_pass(m, p, 512, 2, noise=gpu.PCA, pca=pl, salt_base=5, R=2, n_points=2048)
    assert np.all(np.isfinite(lv)) and np.all(np.abs(lv[:, 0] / 2048) < 0.05)   # the level difference is small
    pl.close()
