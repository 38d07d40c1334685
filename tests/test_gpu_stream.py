"""The normals / increments the fused pass kernel actually consumed (warp-transposed
generation, bridge windows, Philox blocks) compared with the reference stream."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_steps,model", [(256, "gbm"), (50, "heston"), (7, "gbm"), (33, "gbm")])
@pytest.mark.parametrize("offset", [0, 37, (1 << 22) - 3])
def test_fused_sobol_normals_bit_exact(gpu, n_steps, model, offset):
    m = gpu.gbm() if model == "gbm" else gpu.heston()
    D = n_steps * gpu.noise_dim(m)
    R, n = 2, 70
    dump = gpu.debug_pass_dump(m, n_steps, gpu.RAW, use_sobol=True, salt_base=42, R=R, offset=offset, n_points=n)
    for r in range(R):
        ref = gpu.sobol_hh_normal(42 + r, 0, D, offset, n)          # [D, n]
        assert np.array_equal(dump[r], ref.T), (r, np.argwhere(dump[r] != ref.T)[:3])


@pytest.mark.parametrize("N", [1, 4, 16, 32, 64, 256, 512])
def test_fused_bridge_increments(gpu, orc, N):
    T = 1.0
    bb = gpu.bb_create(N, T)
    R, n, off = 2, 64, 100
    dump = gpu.debug_pass_dump(gpu.gbm(T=T), N, gpu.BB, bb=bb, use_sobol=True, salt_base=50, R=R, offset=off,
                               n_points=n)
    for r in range(R):
        z = gpu.sobol_hh_normal(50 + r, 0, N, off, n).astype(np.float64)   # [N, n] in dimension order
        for i in range(0, n, 7):
            ref = orc.bb_apply(N, T, z[:, i])
            assert np.allclose(dump[r, i], ref, atol=3e-6, rtol=1e-5), (r, i)
    bb.close()


def test_fused_philox_normals(gpu, orc):
    m = gpu.heston()
    n_steps, n, first = 19, 50, 1000
    dump = gpu.debug_pass_dump(m, n_steps, gpu.RAW, use_sobol=False, seed=123, salt_base=7, R=2, offset=first,
                               n_points=n)
    D = 2 * n_steps
    for r in range(2):
        for i in range(0, n, 5):
            ref = orc.philox_normals(123, 7 + r, first + i, D)
            assert np.allclose(dump[r, i], ref, atol=2e-5, rtol=2e-5), (r, i)


@pytest.mark.parametrize("model,n_steps,R,n,offset", [("gbm", 32, 2, 1 << 20, 5), ("heston", 32, 3, 700000, 1 << 21)])
def test_carried_start_words_give_the_same_normals(gpu, model, n_steps, R, n, offset):
    """Items of several 32-point groups carry each tile's Sobol start word from group to group in
    shared memory instead of walking it from the digital shift: over a range that splits into
    items of two or more groups, every normal of every replica equals the stream generator's."""
    m = gpu.gbm() if model == "gbm" else gpu.heston()
    D = n_steps * gpu.noise_dim(m)
    dump = gpu.debug_pass_dump(m, n_steps, gpu.RAW, use_sobol=True, salt_base=11, R=R, offset=offset, n_points=n)
    gpi, carry = gpu.debug_last_pass_layout()
    assert gpi >= 2 and carry == 32 * ((D + 31) // 32), (gpi, carry)
    for r in range(R):
        ref = gpu.sobol_hh_normal(11 + r, 0, D, offset, n)
        assert np.array_equal(dump[r], ref.T), (r, np.argwhere(dump[r] != ref.T)[:3])


@pytest.mark.parametrize("N", [16, 64])
def test_carried_start_words_bridge(gpu, orc, N):
    """The bridge's skeleton and window tiles carry their start words too (one slot per tile):
    increments at points spread over a range of multi-group items match the oracle's bridge."""
    T = 1.0
    bb = gpu.bb_create(N, T)
    R, n, off = 2, 700000, 3
    dump = gpu.debug_pass_dump(gpu.gbm(T=T), N, gpu.BB, bb=bb, use_sobol=True, salt_base=21, R=R, offset=off,
                               n_points=n)
    gpi, carry = gpu.debug_last_pass_layout()
    S = N // 32
    assert gpi >= 2 and carry == 32 * (((S + 31) // 32 + S) if N > 32 else 1), (gpi, carry)
    rng = np.random.default_rng(5)
    for r in range(R):
        for i in sorted(rng.choice(n, 24, replace=False)):
            z = gpu.sobol_hh_normal(21 + r, 0, N, off + int(i), 1).astype(np.float64)[:, 0]
            ref = orc.bb_apply(N, T, z)
            assert np.allclose(dump[r, i], ref, atol=3e-6, rtol=1e-5), (r, i)
    bb.close()
