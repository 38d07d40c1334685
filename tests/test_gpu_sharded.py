"""The sharded RQMC driver on one GPU: with the engine's passes as the per-rank compute it is
run_qmc_cuda's result, and replica blocks priced separately (as two ranks would) give the
per-replica sums of one pass over all replicas."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_sharded_qmc_on_the_engine_equals_run_qmc(gpu):
    import fdmc_b200.sharded as sh
    m, p = gpu.gbm(100, 0.03, 0.25, 1.0), gpu.asian(100.0)

    def pass_fn(r0, nr, offset, n):
        return gpu.qmc_pass(m, p, 64, salt_base=42 + r0, R=nr, offset=offset, n_points=n)

    got = sh.run_qmc_sharded(pass_fn, 16, 2e-3, 1 << 10, max_doublings=8)
    ref = gpu.run_qmc(m, p, 2e-3, 64, gpu.qmc_cfg(R=16, N0_per_replica=1 << 10, max_doublings=8))
    assert got["n_samples"] == ref["n_samples"]
    assert abs(got["price"] - ref["price"]) < 1e-12 * abs(ref["price"])
    assert abs(got["std_error"] - ref["std_error"]) < 1e-9 * ref["std_error"]


def test_replica_blocks_reproduce_the_full_pass(gpu):
    m, p = gpu.gbm(100, 0.03, 0.25, 1.0), gpu.asian(100.0)
    full = gpu.qmc_pass(m, p, 64, salt_base=42, R=8, offset=100, n_points=5000)
    a = gpu.qmc_pass(m, p, 64, salt_base=42, R=3, offset=100, n_points=5000)
    b = gpu.qmc_pass(m, p, 64, salt_base=45, R=5, offset=100, n_points=5000)
    np.testing.assert_allclose(np.vstack([a, b]), full, rtol=1e-12)
