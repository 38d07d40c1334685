"""Scrambled-Sobol stream on the GPU vs the oracle: integers bit-exact, normals to the inverse
normal's precision, and the u = 1 edge (methods_cuda.cu:823) in both modes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OFFSETS = [0, 1, (1 << 14) - 1, (1 << 22) - 1, (1 << 32) - (1 << 10)]


@pytest.mark.parametrize("salt", [42, 43, 42 + 16 * 3 + 5, 73])
@pytest.mark.parametrize("offset", OFFSETS)
def test_integers_bit_exact(gpu, orc, salt, offset):
    n = 1024 if offset == OFFSETS[-1] else 777
    for dim0, nd in ((0, 40), (200, 56), (480, 32), (19990, 10)):
        a = gpu.sobol_hh_u32(salt, dim0, nd, offset, n)
        b = orc.sobol_hh_u32(salt, dim0, nd, offset, n)
        assert np.array_equal(a, b), (salt, offset, dim0)


@pytest.mark.parametrize("salt", [42, 59])
def test_normals_match_as241(gpu, orc, salt):
    # CUDA normcdfinvf vs the FP64 AS241 of the same single-precision u: tolerance of the function
    g = gpu.sobol_hh_normal(salt, 0, 64, 1000, 2048).astype(np.float64)
    o = orc.sobol_hh_normal(salt, 0, 64, 1000, 2048)
    assert np.all(np.isfinite(g))
    assert np.max(np.abs(g - o) / (1 + np.abs(o))) < 2e-6


def _find_top_point(orc, salt=42, n=1 << 20):
    for dim in range(64):
        x = orc.sobol_hh_u32(salt, dim, 1, 0, n)[0]
        hit = np.nonzero(x >= 0xFFFFFF80)[0]
        if len(hit):
            return dim, int(hit[0])
    raise AssertionError("no top-edge point found")


def test_u_equals_one_edge(gpu, orc):
    dim, i = _find_top_point(orc)
    compat = gpu.sobol_hh_normal(42, dim, 1, i, 1, flags=gpu.FLAG_COMPAT_U_INF)[0, 0]
    clamp = gpu.sobol_hh_normal(42, dim, 1, i, 1, flags=0)[0, 0]
    assert np.isposinf(compat)                        # the reference's behaviour
    assert np.isfinite(clamp) and 5.0 < clamp < 5.5   # normcdfinvf(1 - 2^-24)
