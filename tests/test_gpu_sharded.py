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


@pytest.mark.parametrize("blocks", [1, 2, 4])
def test_sharded_mlqmc_on_the_engine_agrees_with_run_mlqmc(gpu, blocks):
    """The sharded MLQMC driver with the engine's coupled level passes as the per-rank compute, the
    replicas of every level priced in `blocks` separate launches as that many ranks would: it takes
    the points of mcq_run_mlqmc (salts 42 + l R + r, shared offsets), so its price agrees with the
    driver's to the FP64 summation order of the work items, within 3 standard errors in any case."""
    import fdmc_b200.sharded as sh
    m, p = gpu.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0), gpu.european(100.0, 0.02, 1.0)
    R, M, eps = 16, 4, 5e-3

    def level_fn(l, r0, nr, offset, n):
        out = []
        for k in range(blocks):   # the block split into `blocks` launches
            a = r0 + nr * k // blocks
            b = r0 + nr * (k + 1) // blocks
            if b > a:
                out.append(gpu.level_pass(m, p, 4 * M ** l, M if l else 0, use_sobol=True, salt_base=42 + l * R + a,
                                          R=b - a, offset=offset, n_points=n))
        return np.vstack(out)

    got = sh.run_mlqmc_sharded(level_fn, R, eps, M=M, max_L=6, pilot_n=1000)
    ref = gpu.run_mlqmc(m, p, eps, gpu.mlmc_cfg(M=M, n0_steps=4, max_L=6, pilot_n=1000), gpu.qmc_cfg(R=R))
    assert got["levels"] == ref["levels"]
    assert abs(got["price"] - ref["price"]) < 3 * np.hypot(got["std_error"], ref["std_error"]), (got, ref)
    assert abs(got["price"] - ref["price"]) < 1e-6 * abs(ref["price"]) or got["n_samples"] != ref["n_samples"]
