"""The CPU oracle pinned against published known answers and independent references.

Pins: Black–Scholes known answers printed by the reference (informes_finales/informe_final.txt:7,
:158); scipy.special.ndtri for the AS241 inverse normal; Random123 known-answer vectors for
Philox4x32-10; numpy.linalg.eigh for the PCA factor; the literal Hong–Hickernell scramble
(hh_scramble row by row, methods_cuda.cu:781-795) for the fast pre-scrambled form.  The
reference's own Sobol-HH integers and normals are pinned in test_golden.py.
"""
import numpy as np
import pytest
import scipy.special as sp


def test_bs_known_answers(orc):
    # informe_final.txt:7 and :158
    assert abs(orc.bs_call(100, 100, 1, 0.05, 0.2) - 10.450584) < 5e-7
    assert abs(orc.bs_call(100, 180, 1, 0.05, 0.2) - 0.028643) < 5e-7


def test_ppnd16_matches_scipy(orc):
    ps = np.concatenate([np.linspace(1e-12, 1 - 1e-12, 4001), [2.3283064365386963e-10, 0.5, 0.025, 0.975]])
    got = np.array([orc.ppnd16(p) for p in ps])
    ref = sp.ndtri(ps)
    assert np.max(np.abs(got - ref) / np.maximum(1, np.abs(ref))) < 1e-14


def test_philox_known_answers(orc):
    # Random123 kat_vectors, philox4x32_10
    kat = [
        ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
        ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
        ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
         [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
    ]
    for ctr, key, want in kat:
        assert orc.philox(ctr, key) == want


@pytest.mark.parametrize("m", [1, 2, 7, 64, 256])
def test_pca_closed_form(orc, m):
    T = 1.0
    M = orc.pca_matrix(m, T)
    h = T / m
    C = h * np.minimum.outer(np.arange(1, m + 1), np.arange(1, m + 1)).astype(float)
    Mc = np.cumsum(M, axis=0)                       # M_cum = V sqrt(lambda)
    assert np.allclose(Mc @ Mc.T, C, atol=1e-12 * m)
    lam = np.sort(np.linalg.eigvalsh(C))[::-1]
    assert np.allclose((Mc ** 2).sum(axis=0), lam, rtol=1e-10)
    assert np.all(np.diff((Mc ** 2).sum(axis=0)) <= 1e-12)   # descending
    assert np.all(Mc[0] > 0)                          # sign convention: first component positive
    if m <= 64:
        assert np.allclose(orc.pca_matrix(m, T, jacobi=True), M, atol=1e-10)


@pytest.mark.parametrize("N", [1, 2, 8, 64, 256])
def test_bridge_is_exact_brownian(orc, N):
    T = 1.3
    B = np.stack([orc.bb_apply(N, T, e) for e in np.eye(N)], axis=1)   # dW = B z
    assert np.allclose(B @ B.T, (T / N) * np.eye(N), atol=1e-12)
    mi, li, ri, wl, wr, sd = orc.bb_tables(N, T)
    assert mi[0] == N and abs(sd[0] - np.sqrt(T)) < 1e-15
    if N > 1:
        assert mi[1] == N // 2 and li[1] == 0 and ri[1] == N


def test_scramble_fast_equals_literal(orc):
    for salt in (42, 43, 42 + 16 * 3 + 5, 0xFFFFFFFF):
        for dim0, nd in ((0, 3), (255, 2), (19990, 10)):
            for off in (0, 1, 12345, (1 << 22) - 1, (1 << 32) - 1024):
                a = orc.sobol_hh_u32(salt, dim0, nd, off, 40)
                b = orc.sobol_hh_u32(salt, dim0, nd, off, 40, literal=True)
                assert np.array_equal(a, b)


def test_scramble_row_aliasing_is_reproduced(orc):
    # Row seeds are splitmix32(base ^ k) with base = splitmix32(salt) ^ dim (methods_cuda.cu:786,819):
    # rows (dim, k) and (dim ^ j, k ^ j) coincide.  The restatement must keep that structure.
    base = orc.splitmix32(42)
    for dim, j in ((5, 3), (100, 17)):
        for k in range(8):
            assert orc.splitmix32((base ^ dim) ^ k) == orc.splitmix32((base ^ (dim ^ j)) ^ (k ^ j))


def test_u_mapping_top_edge(orc):
    # methods_cuda.cu:823: u = ((float)s + 1) * 2^-32 rounds to 1.0f for s >= 0xFFFFFF80
    assert orc.u_of(0xFFFFFF7F, 1) < 1.0
    assert orc.u_of(0xFFFFFF80, 1) == 1.0
    assert orc.u_of(0xFFFFFFFF, 1) == 1.0
    assert orc.u_of(0xFFFFFFFF, 0) == np.float32(1.0) - np.float32(2.0 ** -24)
    assert orc.u_of(0, 0) == np.float32(2.0 ** -32)


def test_geometric_asian_closed_form_vs_oracle_qmc(orc):
    T = orc.T
    m, p = T.gbm(100.0, 0.05, 0.2, 1.0), T.geom_asian(100.0)
    n = 64
    nz = orc.noise(T.BB, n, 1.0)
    s = orc.qmc_sums(m, p, n, nz, R=8, N=4096)
    means = s[:, 0] / 4096
    est, se = means.mean(), means.std(ddof=1) / np.sqrt(len(means))
    ref = orc.geom_asian(100.0, 100.0, 1.0, 0.05, 0.2, n)
    assert abs(est - ref) < 4 * se + 0.02          # Euler bias at 64 steps is ~1e-2


def test_down_out_closed_form_limits(orc):
    # B -> 0 recovers the vanilla call; B = S0 knocks out immediately
    assert abs(orc.down_out_call(100, 100, 1e-6, 1, 0.05, 0.2) - orc.bs_call(100, 100, 1, 0.05, 0.2)) < 1e-9
    assert orc.down_out_call(100, 100, 100, 1, 0.05, 0.2) == 0.0
    v = orc.down_out_call(100, 100, 80, 1, 0.02, 0.2)
    assert 0 < v < orc.bs_call(100, 100, 1, 0.02, 0.2)


def test_oracle_qmc_sums_independent_of_threads(orc):
    T = orc.T
    m, p = T.heston(rho=-0.7, xi=0.3), T.asian(100.0)
    a = orc.qmc_sums(m, p, 8, None, R=3, offset=7, N=333, threads=1)
    b = orc.qmc_sums(m, p, 8, None, R=3, offset=7, N=333, threads=4)
    assert np.array_equal(a, b)
