"""Edge cases of the fused pass through the C ABI: empty and single-point ranges, the last points
below 2^32, the largest Sobol dimension count, ragged groups, and the range errors."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _close(g, o, N):
    return np.abs(g[:, 0] / N - o[:, 0] / N).max() < 2e-4 * (1 + np.abs(o[:, 0] / N).max())


def test_empty_range_gives_zero_sums(gpu):
    m, p = gpu.gbm(), gpu.asian(100.0)
    s = gpu.qmc_pass(m, p, 64, salt_base=42, R=3, offset=17, n_points=0)
    assert s.shape == (3, 2) and not s.any()


@pytest.mark.parametrize("offset", [0, 31, 32, 1 << 20, (1 << 32) - 1])
def test_single_point(gpu, orc, offset):
    m, p = gpu.gbm(100.0, 0.05, 0.2, 1.0), gpu.european(100.0, 0.05, 1.0)
    g = gpu.qmc_pass(m, p, 32, salt_base=42, R=2, offset=offset, n_points=1)
    o = orc.qmc_sums(m, p, 32, None, salt_base=42, R=2, offset=offset, N=1)
    assert _close(g, o, 1), (g, o)


def test_last_points_below_two_to_the_32(gpu, orc):
    m, p = gpu.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0), gpu.lookback(0.2)
    N = 1000
    off = (1 << 32) - N
    g = gpu.qmc_pass(m, p, 16, salt_base=7, R=2, offset=off, n_points=N)
    o = orc.qmc_sums(m, p, 16, None, salt_base=7, R=2, offset=off, N=N)
    assert _close(g, o, N), (g, o)


def test_largest_dimension_count(gpu, orc):
    """Heston with 10000 steps uses all 20000 Sobol dimensions of the direction table."""
    m, p = gpu.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0), gpu.asian(100.0)
    N = 96
    g = gpu.qmc_pass(m, p, 10000, salt_base=11, R=1, offset=5, n_points=N)
    o = orc.qmc_sums(m, p, 10000, None, salt_base=11, R=1, offset=5, N=N)
    assert _close(g, o, N), (g, o)


def test_ragged_groups_add_up(gpu):
    """A range split at points that are not multiples of the 32-point group gives the same sums
    as the whole range (up to FP64 summation order)."""
    m, p = gpu.gbm(100.0, 0.03, 0.25, 1.0), gpu.asian(100.0)
    whole = gpu.qmc_pass(m, p, 64, salt_base=42, R=2, offset=3, n_points=10007)
    parts = sum(gpu.qmc_pass(m, p, 64, salt_base=42, R=2, offset=a, n_points=b - a)
                for a, b in [(3, 40), (40, 41), (41, 5000), (5000, 10010)])
    np.testing.assert_allclose(parts, whole, rtol=1e-12)


def test_range_errors(gpu):
    m, p = gpu.gbm(), gpu.asian(100.0)
    with pytest.raises(gpu.MCQError) as e:
        gpu.qmc_pass(m, p, 64, salt_base=42, R=1, offset=(1 << 32) - 10, n_points=11)
    assert e.value.code == 4
    h = gpu.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    with pytest.raises(gpu.MCQError) as e:
        gpu.qmc_pass(h, p, 10001, salt_base=42, R=1, n_points=32)   # 20002 dimensions
    assert e.value.code == 4


def test_bounded_wait_reports_timeout_and_the_context_survives(gpu, orc):
    """A bounded device wait that nothing completes gives up, the host reads MCQ_ERR_TIMEOUT from
    the status word, and the next pass runs normally."""
    with pytest.raises(gpu.MCQError) as e:
        gpu.debug_wait_timeout(1000)
    assert e.value.code == 7
    assert b"timed out" in gpu.lib().mcq_last_error()
    m, p = gpu.gbm(100.0, 0.05, 0.2, 1.0), gpu.asian(100.0)
    g = gpu.qmc_pass(m, p, 64, salt_base=42, R=2, offset=3, n_points=2000)
    o = orc.qmc_sums(m, p, 64, None, salt_base=42, R=2, offset=3, N=2000)
    assert _close(g, o, 2000), (g, o)


def test_assisted_pass_at_the_last_points_and_many_dimensions(gpu, orc):
    """An assisted pass (few groups, long paths): Heston with 10000 Sobol dimensions on the last
    3200 points below 2^32."""
    m, p = gpu.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0), gpu.lookback(0.2)
    N = 3200
    off = (1 << 32) - N
    g = gpu.qmc_pass(m, p, 5000, salt_base=3, R=1, offset=off, n_points=N)
    o = orc.qmc_sums(m, p, 5000, None, salt_base=3, R=1, offset=off, N=N)
    assert _close(g, o, N), (g, o)


@pytest.mark.parametrize("R", [1, 32])
def test_packed_pass_at_the_last_points(gpu, orc, R):
    """A packed pass (paths of 3 normals, 10 groups per tile) ending at 2^32, with one and 32 replicas."""
    m, p = gpu.gbm(100.0, 0.05, 0.2, 1.0), gpu.asian(100.0)
    N = 1000
    off = (1 << 32) - N
    g = gpu.qmc_pass(m, p, 3, salt_base=11, R=R, offset=off, n_points=N)
    o = orc.qmc_sums(m, p, 3, None, salt_base=11, R=R, offset=off, N=N)
    assert _close(g, o, N), (g, o)
