"""The engine against the reference's own CUDA outputs (tests/golden/ref_golden.npz):
scrambled integers bit-exact, the fused pass's per-replica sums on the same points to FP32
rounding, and the adaptive drivers within their statistical error."""
import json
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)
import golden_cases  # noqa: E402


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "ref_golden.npz"))


@pytest.fixture(scope="module")
def meta():
    with open(os.path.join(GOLD, "ref_golden.json")) as f:
        return json.load(f)


def test_integers_equal_reference(gpu, gold):
    for s in golden_cases.SALTS:
        for o in golden_cases.OFFSETS:
            for d0, nd in golden_cases.DIMS:
                ref = gold[f"u32_{s}_{o}_{d0}"]
                assert np.array_equal(ref, gpu.sobol_hh_u32(s, d0, nd, o, ref.shape[1])), (s, o, d0)


def test_normals_equal_reference_kernel(gpu, gold):
    # same integers, same u mapping, same CUDA normcdfinvf: the floats are identical
    for o in (0, (1 << 22) - 1):
        ref = gold[f"normal_42_{o}"]
        assert np.array_equal(ref, gpu.sobol_hh_normal(42, 0, 16, o, ref.shape[1]))


NAMES = [c[0] for c in golden_cases.cases(__import__("oracle_py").T) if "pca" not in c[0]]


@pytest.mark.parametrize("name", NAMES)
def test_pass_sums_equal_reference(gpu, gold, name):
    case = {c[0]: c for c in golden_cases.cases(gpu.mcq_types)}[name]
    _, m, p, n_steps, mode, salt0, R, off, N = case
    bb = gpu.bb_create(n_steps, m.T) if mode == gpu.BB else None
    mine = gpu.qmc_pass(m, p, n_steps, noise=mode, bb=bb, salt_base=salt0, R=R, offset=off, n_points=N)
    ref = gold["pass_" + name]
    for r in range(R):
        a, b = ref[r, 0] / N, mine[r, 0] / N
        extra = 60.0 / N if "upout" in name else 0.0
        assert abs(a - b) < 1e-4 * (1 + abs(a)) + extra, (name, r, a, b)
    if bb:
        bb.close()


def test_drivers_agree_with_reference(gpu, meta):
    """The adaptive drivers against the reference's own drivers' results, within 3 standard errors
    of the difference (3 hypot(se_engine, se_reference)).  MC and MLMC draw pseudo-random numbers
    (XORWOW there, Philox here), MLQMC the same scrambled points."""
    d = meta["drivers"]
    gbm, eur = gpu.gbm(100.0, 0.05, 0.2, 1.0), gpu.european(100.0, 0.05, 1.0)
    mc = gpu.run_mc(gbm, eur, 1e-2, 64)
    ref = d["mc_gbm_eur_64_eps1e-2"]
    assert abs(mc["price"] - ref[0]) < 3 * np.hypot(mc["std_error"], ref[1]), (mc, ref)
    ml = gpu.run_mlmc(gbm, eur, 1e-2, gpu.mlmc_cfg(M=2, max_L=10, pilot_n=400))
    ref = d["mlmc_gbm_eur_eps1e-2"]
    assert abs(ml["price"] - ref[0]) < 3 * np.hypot(ml["std_error"], ref[1]), (ml, ref)
    q = gpu.run_mlqmc(gbm, eur, 5e-3, gpu.mlmc_cfg(M=2, max_L=10, pilot_n=400), gpu.qmc_cfg(R=16))
    ref = d["mlqmc_gbm_eur_eps5e-3"]
    assert abs(q["price"] - ref[0]) < 3 * np.hypot(q["std_error"], ref[1]), (q, ref)
    hes = gpu.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    h = gpu.run_mlqmc(hes, gpu.european(100.0, 0.02, 1.0), 1e-2, gpu.mlmc_cfg(M=4, max_L=8, pilot_n=400),
                      gpu.qmc_cfg(R=16))
    ref = d["mlqmc_heston_eur_M4_eps1e-2"]
    assert abs(h["price"] - ref[0]) < 3 * np.hypot(h["std_error"], ref[1]), (h, ref)


@pytest.fixture(scope="module")
def gold_levels():
    return np.load(os.path.join(GOLD, "ref_golden_levels.npz"))


@pytest.fixture(scope="module")
def meta_levels():
    with open(os.path.join(GOLD, "ref_golden_levels.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", [c[0] for c in golden_cases.level_cases(__import__("oracle_py").T)])
def test_level_pass_equals_reference_kernel(gpu, gold_levels, meta_levels, name):
    """The fused coupled level pass against the reference's own kernel_mlmc (methods_cuda.cu:445-518)
    on the same scrambled points: per-replica means of dY and Yf to FP32 rounding.  Heston
    lookback under MCQ_FLAG_COMPAT_HESTON_MLMC, which reproduces the reference's skipped running
    update (:464-490)."""
    case = {c[0]: c for c in golden_cases.level_cases(gpu.mcq_types)}[name]
    _, m, p, level, M, _, R, off, N = case
    info = {c["name"]: c for c in meta_levels["levels"]}[name]
    flags = gpu.FLAG_COMPAT_HESTON_MLMC if "heston_lookback" in name else 0
    mine = gpu.level_pass(m, p, M ** level, M if level else 0, use_sobol=True, salt_base=info["salt0"], R=R,
                          offset=off, n_points=N, flags=flags)
    ref = gold_levels[name]
    for r in range(R):
        scale = 1 + abs(ref[r, 2] / N)
        extra = 60.0 / N if "upout" in name else 0.0
        for k in (0, 2):
            assert abs(ref[r, k] / N - mine[r, k] / N) < 1e-4 * scale + extra, (name, r, k, ref[r], mine[r])


@pytest.mark.parametrize("name", [c[0] for c in golden_cases.is_cases(__import__("oracle_py").T)])
def test_is_pass_equals_reference_kernel(gpu, gold_levels, meta_levels, name):
    """The fused importance-sampling pass against the reference's kernel_is_gbm
    (methods_cuda.cu:685-707) on the same scrambled points."""
    case = {c[0]: c for c in golden_cases.is_cases(gpu.mcq_types)}[name]
    _, m, p, n_steps, _, _, R, off, N = case
    info = {c["name"]: c for c in meta_levels["is"]}[name]
    mine = gpu.is_pass(m, p, n_steps, info["z_step"], use_sobol=True, salt_base=info["salt0"], R=R, offset=off,
                       n_points=N)
    ref = gold_levels[name]
    for r in range(R):
        assert abs(ref[r, 0] / N - mine[r, 0] / N) < 1e-4 * (1 + abs(ref[r, 0] / N)), (name, r, ref[r], mine[r])
