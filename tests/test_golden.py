"""The CPU oracle against outputs of the reference's own CUDA code (tests/golden/ref_golden.npz,
written on a B200 by tests/golden/make_ref_golden.py from oracle/_ref, the reference built from
its sources).  Integers bit-exact; normals to the inverse normal's precision; per-replica sums
of the reference's generate -> transform -> price steps to FP32 rounding (the oracle steps in
FP64 on the same points)."""
import json
import os
import sys

import numpy as np
import pytest

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


def test_reference_integers_equal_oracle(orc, gold):
    n = 0
    for s in golden_cases.SALTS:
        for o in golden_cases.OFFSETS:
            for d0, nd in golden_cases.DIMS:
                ref = gold[f"u32_{s}_{o}_{d0}"]
                assert np.array_equal(ref, orc.sobol_hh_u32(s, d0, nd, o, ref.shape[1])), (s, o, d0)
                assert np.array_equal(ref, orc.sobol_hh_u32(s, d0, nd, o, ref.shape[1], literal=True))
                n += ref.size
    assert n == 4 * 5 * 3 * 16 * 32


def test_reference_normals_match_oracle(orc, gold):
    for o in (0, (1 << 22) - 1):
        ref = gold[f"normal_42_{o}"].astype(np.float64)
        mine = orc.sobol_hh_normal(42, 0, 16, o, ref.shape[1])
        assert np.max(np.abs(ref - mine) / (1 + np.abs(mine))) < 2e-6


@pytest.mark.parametrize("name", [c[0] for c in golden_cases.cases(__import__("oracle_py").T)])
def test_reference_pass_sums_match_oracle(orc, gold, meta, name):
    case = {c[0]: c for c in golden_cases.cases(orc.T)}[name]
    _, m, p, n_steps, mode, salt0, R, off, N = case
    info = {c["name"]: c for c in meta["cases"]}[name]
    assert info["top_edge_hits"] == 0
    ref = gold["pass_" + name]
    nz = None if mode == orc.T.RAW else orc.noise(mode, n_steps, m.T)
    mine = orc.qmc_sums(m, p, n_steps, nz, salt0, R, off, N)
    tol = 2e-4 if mode != orc.T.PCA else 5e-4
    for r in range(R):
        a, b = ref[r, 0] / N, mine[r, 0] / N
        extra = 60.0 / N if "upout" in name else 0.0
        assert abs(a - b) < tol * (1 + abs(b)) + extra, (name, r, a, b)


@pytest.fixture(scope="module")
def gold_levels():
    return np.load(os.path.join(GOLD, "ref_golden_levels.npz"))


@pytest.fixture(scope="module")
def meta_levels():
    with open(os.path.join(GOLD, "ref_golden_levels.json")) as f:
        return json.load(f)


LEVEL_NAMES = [c[0] for c in golden_cases.level_cases(__import__("oracle_py").T)]
IS_NAMES = [c[0] for c in golden_cases.is_cases(__import__("oracle_py").T)]


@pytest.mark.parametrize("name", LEVEL_NAMES)
def test_reference_level_sums_match_oracle(orc, gold_levels, meta_levels, name):
    """The reference's coupled level kernel (kernel_mlmc, methods_cuda.cu:445-518) against the
    oracle's coupled pair on the same points: dY and Yf means to FP32 rounding of the payoff.
    The reference's Heston level kernel skips the running update (:464-490), so its lookback is
    compared with the oracle under MCQ_FLAG_COMPAT_HESTON_MLMC."""
    case = {c[0]: c for c in golden_cases.level_cases(orc.T)}[name]
    _, m, p, level, M, _, R, off, N = case
    info = {c["name"]: c for c in meta_levels["levels"]}[name]
    flags = orc.T.FLAG_COMPAT_HESTON_MLMC if "heston_lookback" in name else 0
    mine = orc.level_sums(m, p, M ** level, M if level else 0, None, use_sobol=True, salt_base=info["salt0"], R=R,
                          offset=off, N=N, flags=flags)
    ref = gold_levels[name]
    for r in range(R):
        scale = 1 + abs(ref[r, 2] / N)
        extra = 60.0 / N if "upout" in name else 0.0
        for k in (0, 2):
            assert abs(ref[r, k] / N - mine[r, k] / N) < 2e-4 * scale + extra, (name, r, k, ref[r], mine[r])


@pytest.mark.parametrize("name", IS_NAMES)
def test_reference_is_sums_match_oracle(orc, gold_levels, meta_levels, name):
    """The reference's importance-sampling kernel (kernel_is_gbm, methods_cuda.cu:685-707) against
    the oracle's restatement on the same scrambled points: mean and second moment of the weighted
    payoff."""
    case = {c[0]: c for c in golden_cases.is_cases(orc.T)}[name]
    _, m, p, n_steps, _, _, R, off, N = case
    info = {c["name"]: c for c in meta_levels["is"]}[name]
    mine = orc.is_sums(m, p, n_steps, info["z_step"], use_sobol=True, salt_base=info["salt0"], R=R, offset=off, N=N)
    ref = gold_levels[name]
    for r in range(R):
        assert abs(ref[r, 0] / N - mine[r, 0] / N) < 2e-4 * (1 + abs(mine[r, 0] / N)), (name, r, ref[r], mine[r])
        assert abs(ref[r, 1] - mine[r, 1]) < 1e-3 * (1 + abs(mine[r, 1])), (name, r, ref[r], mine[r])
