"""ctypes binding of the CPU oracle (oracle/liboracle.so).  TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference leg as the
checker or the timed CPU baseline; the product engine never imports it.
"""
import ctypes as C
import importlib.util
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "liboracle.so")


def _types():
    name = "fdmc_b200_types"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(ROOT, "financial-derivatives-montecarlo_b200", "mcq_types.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


T = _types()
_P = C.POINTER
_pd = _P(C.c_double)
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_ppnd16.restype = C.c_double
        L.orc_ppnd16.argtypes = [C.c_double]
        for f in ("orc_bs_call", "orc_geom_asian", "orc_down_out_call"):
            getattr(L, f).restype = C.c_double
        L.orc_bs_call.argtypes = [C.c_double] * 5
        L.orc_geom_asian.argtypes = [C.c_double] * 5 + [C.c_int]
        L.orc_down_out_call.argtypes = [C.c_double] * 6
        L.orc_splitmix32.restype = C.c_uint32
        L.orc_splitmix32.argtypes = [C.c_uint32]
        L.orc_hh_scramble.restype = C.c_uint32
        L.orc_hh_scramble.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_u_of.restype = C.c_float
        L.orc_u_of.argtypes = [C.c_uint32, C.c_int]
        L.orc_path_payoff.restype = C.c_double
        L.orc_path_payoff_f.restype = C.c_double
        L.orc_basket_level_f.restype = C.c_double
        L.orc_is_payoff.restype = C.c_double
        L.orc_level_payoff.restype = C.c_double
        _lib = L
    return _lib


class Noise(C.Structure):
    _fields_ = [("mode", C.c_int), ("N", C.c_int),
                ("map_idx", _P(C.c_int)), ("left_idx", _P(C.c_int)), ("right_idx", _P(C.c_int)),
                ("wl", _pd), ("wr", _pd), ("sd", _pd), ("M_pca", _pd), ("pca_fp16", C.c_int)]


def bb_tables(N, T_):
    mi, li, ri = (np.zeros(N, np.int32) for _ in range(3))
    wl, wr, sd = (np.zeros(N, np.float64) for _ in range(3))
    rc = lib().orc_bb_precompute(C.c_int(N), C.c_double(T_), mi.ctypes.data_as(_P(C.c_int)),
                                 li.ctypes.data_as(_P(C.c_int)), ri.ctypes.data_as(_P(C.c_int)),
                                 wl.ctypes.data_as(_pd), wr.ctypes.data_as(_pd), sd.ctypes.data_as(_pd))
    assert rc == 0
    return mi, li, ri, wl, wr, sd


def pca_matrix(m, T_, jacobi=False):
    M = np.zeros(m * m)
    f = lib().orc_pca_jacobi if jacobi else lib().orc_pca_compute
    assert f(C.c_int(m), C.c_double(T_), M.ctypes.data_as(_pd)) == 0
    return M.reshape(m, m).T  # M[i, k]


def noise(mode, N=0, T_=1.0, pca_fp16=True):
    """orc_noise for RAW / BB / PCA; keeps its arrays alive on the returned object."""
    nz = Noise()
    nz.mode, nz.N = mode, N
    keep = []
    if mode == T.BB:
        mi, li, ri, wl, wr, sd = bb_tables(N, T_)
        keep += [mi, li, ri, wl, wr, sd]
        nz.map_idx, nz.left_idx, nz.right_idx = (a.ctypes.data_as(_P(C.c_int)) for a in (mi, li, ri))
        nz.wl, nz.wr, nz.sd = (a.ctypes.data_as(_pd) for a in (wl, wr, sd))
    elif mode == T.PCA:
        M = np.ascontiguousarray(pca_matrix(N, T_).T.reshape(-1))  # column-major
        keep.append(M)
        nz.M_pca = M.ctypes.data_as(_pd)
        nz.pca_fp16 = int(pca_fp16)
    nz._keep = keep
    return nz


def ppnd16(p):
    return lib().orc_ppnd16(float(p))


def bs_call(S0, K, T_, r, sigma):
    return lib().orc_bs_call(S0, K, T_, r, sigma)


def geom_asian(S0, K, T_, mu, sigma, n):
    return lib().orc_geom_asian(S0, K, T_, mu, sigma, n)


def down_out_call(S0, K, B, T_, r, sigma):
    return lib().orc_down_out_call(S0, K, B, T_, r, sigma)


def splitmix32(x):
    return lib().orc_splitmix32(x)


def hh_scramble(raw, base):
    return lib().orc_hh_scramble(raw, base)


def u_of(s, flags=0):
    return lib().orc_u_of(s, flags)


def philox(ctr, key):
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10((C.c_uint32 * 4)(*ctr), (C.c_uint32 * 2)(*key), o)
    return list(o)


def philox_normals(seed, stream, path, n):
    z = np.zeros(n)
    lib().orc_philox_normals(C.c_uint32(seed), C.c_uint32(stream), C.c_uint64(path), C.c_int(n), z.ctypes.data_as(_pd))
    return z


def sobol_hh_u32(salt, dim0, nd, offset, n, literal=False):
    out = np.zeros((nd, n), np.uint32)
    f = lib().orc_sobol_hh_u32_literal if literal else lib().orc_sobol_hh_u32
    f(C.c_uint32(salt), C.c_int(dim0), C.c_int(nd), C.c_uint32(offset), C.c_int64(n),
      out.ctypes.data_as(_P(C.c_uint32)))
    return out


def sobol_hh_normal(salt, dim0, nd, offset, n, flags=0):
    out = np.zeros((nd, n))
    lib().orc_sobol_hh_normal(C.c_uint32(salt), C.c_int(dim0), C.c_int(nd), C.c_uint32(offset), C.c_int64(n),
                              C.c_int(flags), out.ctypes.data_as(_pd))
    return out


def path_payoff(m, p, n_steps, z, nz=None, flags=0):
    z = np.ascontiguousarray(z, dtype=np.float64)
    return lib().orc_path_payoff_f(C.byref(m), C.byref(p), C.c_int(n_steps), C.byref(nz) if nz else None,
                                   z.ctypes.data_as(_pd), C.c_int(flags))


def qmc_sums(m, p, n_steps, nz=None, salt_base=42, R=1, offset=0, N=1024, flags=0, threads=0):
    out = np.zeros((R, 2))
    rc = lib().orc_qmc_sums(C.byref(m), C.byref(p), C.c_int(n_steps), C.byref(nz) if nz else None,
                            C.c_uint32(salt_base), C.c_int(R), C.c_uint32(offset), C.c_int64(N), C.c_int(flags),
                            C.c_int(threads), out.ctypes.data_as(_pd))
    assert rc == 0, rc
    return out


def level_sums(m, p, n_fine, M, nz=None, use_sobol=True, seed=42, salt_base=42, R=1, offset=0, N=1024, flags=0,
               threads=0):
    out = np.zeros((R, 4))
    rc = lib().orc_level_sums(C.byref(m), C.byref(p), C.c_int(n_fine), C.c_int(M), C.byref(nz) if nz else None,
                              C.c_int(int(use_sobol)), C.c_uint32(seed), C.c_uint32(salt_base), C.c_int(R),
                              C.c_uint32(offset), C.c_int64(N), C.c_int(flags), C.c_int(threads),
                              out.ctypes.data_as(_pd))
    assert rc == 0, rc
    return out


def basket_level(m, p, n_fine, M, z, flags=0):
    """One coupled basket path pair (GBM or Dupire basket): (Yf, Yc, dd[n_assets]); M <= 0 is
    level 0."""
    z = np.ascontiguousarray(z, dtype=np.float64)
    dd = np.zeros(m.n_assets)
    yc = C.c_double()
    L = lib()
    L.orc_basket_level_f.restype = C.c_double
    yf = L.orc_basket_level_f(C.byref(m), C.byref(p), C.c_int(n_fine), C.c_int(M), z.ctypes.data_as(_pd),
                              C.byref(yc), dd.ctypes.data_as(_pd), C.c_int(flags))
    return yf, yc.value, dd


def basket_level_sums(m, p, n_fine, M, salt_base=42, R=1, offset=0, N=1024, flags=0, threads=0):
    out = np.zeros((R, 4 + m.n_assets))
    rc = lib().orc_basket_level_sums(C.byref(m), C.byref(p), C.c_int(n_fine), C.c_int(M), C.c_uint32(salt_base),
                                     C.c_int(R), C.c_uint32(offset), C.c_int64(N), C.c_int(flags), C.c_int(threads),
                                     out.ctypes.data_as(_pd))
    assert rc == 0, rc
    return out


def is_sums(m, p, n_steps, z_star, use_sobol=True, seed=42, salt_base=42, R=1, offset=0, N=1024, flags=0,
            threads=0):
    """kernel_is_gbm in FP64 (z_star: the per-step shift); sums[R][2] = {sum Y, sum Y^2}."""
    out = np.zeros((R, 2))
    rc = lib().orc_is_sums(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_double(z_star), C.c_int(int(use_sobol)),
                           C.c_uint32(seed), C.c_uint32(salt_base), C.c_int(R), C.c_uint32(offset), C.c_int64(N),
                           C.c_int(flags), C.c_int(threads), out.ctypes.data_as(_pd))
    assert rc == 0, rc
    return out


def mc_sums(m, p, n_steps, seed, stream, first_path, n_paths, threads=0):
    out = np.zeros(2)
    lib().orc_mc_sums(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_uint32(seed), C.c_uint32(stream),
                      C.c_int64(first_path), C.c_int64(n_paths), C.c_int(threads), out.ctypes.data_as(_pd))
    return out


def run_qmc(m, p, eps, n_steps, nz=None, R=32, max_doublings=20, N0=1 << 14, salt_base=42, flags=0, threads=0):
    r = T.Result()
    rc = lib().orc_run_qmc(C.byref(m), C.byref(p), C.c_double(eps), C.c_int(n_steps), C.byref(nz) if nz else None,
                           C.c_int(R), C.c_int(max_doublings), C.c_int64(N0), C.c_uint32(salt_base), C.c_int(flags),
                           C.c_int(threads), C.byref(r))
    assert rc == 0, rc
    return r.as_dict()


def max_threads():
    return lib().orc_max_threads()


def bb_apply(N, T_, z):
    """One path of the oracle bridge: z (BFS order) -> time-ordered increments."""
    mi, li, ri, wl, wr, sd = bb_tables(N, T_)
    z = np.ascontiguousarray(z, dtype=np.float64)
    dW = np.zeros(N)
    lib().orc_bb_apply(C.c_int(N), mi.ctypes.data_as(_P(C.c_int)), li.ctypes.data_as(_P(C.c_int)),
                       ri.ctypes.data_as(_P(C.c_int)), wl.ctypes.data_as(_pd), wr.ctypes.data_as(_pd),
                       sd.ctypes.data_as(_pd), z.ctypes.data_as(_pd), dW.ctypes.data_as(_pd))
    return dW


def run_mlqmc(m, p, eps, M=2, max_L=8, n0=1, pilot_n=1000, R=16, salt_base=42, flags=0, threads=0,
              basket=False, max_iter=50):
    """MLQMC adaptive driver in FP64 on the oracle's coupled level sums: the arithmetic of
    run_mlqmc_cuda (methods_cuda.cu:1680-2016) — pilots on levels 0..2, N_opt =
    ceil(2 / (R eps^2) sqrt(sig2_l / C_l) sum_k sqrt(sig2_k C_k)) with N_opt >= 100, merge of
    the extra samples, bias test max(|E_L|, |E_{L-1}|) / (M - 1) < eps / sqrt(2), a new level
    from its pilot, 50 iterations at most.  Level l uses salts salt_base + l R + r (Sobol while
    its n0 M^l x factors dimensions fit the 20000-dimension table, Philox key salt_base and
    stream salt_base + l R + r beyond).  basket=True runs the correlated GBM basket pair
    (orc_basket_level_sums) and also returns the per-asset pathwise deltas."""
    nd = m.n_assets if basket else (2 if m.kind == T.HESTON else 1)
    E = [0.0] * (max_L + 1)
    sig2 = [0.0] * (max_L + 1)
    Nl = [0] * (max_L + 1)
    off = [0] * (max_L + 1)
    dl = [np.zeros(nd) for _ in range(max_L + 1)]
    ps = [0.0]

    def nfine(l):
        return n0 * M ** l

    def level(l, n):
        nf = nfine(l)
        salt = salt_base + l * R
        if basket:
            s = basket_level_sums(m, p, nf, M if l else 0, salt_base=salt, R=R, offset=off[l], N=n, flags=flags,
                                  threads=threads)
        else:
            sob = nf * nd <= 20000
            s = level_sums(m, p, nf, M if l else 0, None, use_sobol=sob, seed=salt_base, salt_base=salt, R=R,
                           offset=off[l], N=n, flags=flags, threads=threads)
        off[l] += n
        ps[0] += R * n * (nf + (nf // M if l else 0))
        rm = s[:, 0] / n
        mm = rm.mean()
        v = ((rm - mm) ** 2).sum() / (R - 1) if R > 1 else 0.0
        d = (s[:, 4:4 + nd] / n).mean(axis=0) if basket else np.zeros(nd)
        return mm, v, d

    def absorb(l, n, res):
        mm, v, d = res
        if Nl[l] == 0:
            E[l], sig2[l], dl[l] = mm, v * n, d
        else:
            wo, wn = float(Nl[l]), float(n)
            E[l] = (E[l] * wo + mm * wn) / (wo + wn)
            sig2[l] = (sig2[l] * wo + v * wn * wn) / (wo + wn)
            dl[l] = (dl[l] * wo + d * wn) / (wo + wn)
        Nl[l] += n

    L = 2
    for l in range(L + 1):
        absorb(l, pilot_n, level(l, pilot_n))
    converged, it = False, 0
    while not converged and L <= max_L and it < max_iter:
        it += 1
        st = sum(np.sqrt(sig2[l] * M ** l) for l in range(L + 1))
        for l in range(L + 1):
            nopt = max(int(np.ceil(2.0 / (R * eps * eps) * np.sqrt(sig2[l] / M ** l) * st)), 100)
            if nopt > Nl[l]:
                absorb(l, nopt - Nl[l], level(l, nopt - Nl[l]))
        bias = abs(E[L]) / max(M - 1, 1)
        if L >= 1:
            bias = max(bias, abs(E[L - 1]) * M / max(M * (M - 1), 1))
        converged = bias < eps / np.sqrt(2.0)
        if not converged and L < max_L:
            L += 1
            absorb(L, pilot_n, level(L, pilot_n))
    price = sum(E[:L + 1])
    se = float(np.sqrt(sum(sig2[l] / (Nl[l] * R) for l in range(L + 1))))
    return {"price": price, "std_error": se, "levels": L + 1, "converged": converged,
            "n_samples": int(sum(Nl[:L + 1]) * R), "path_steps": ps[0],
            "delta": sum(dl[:L + 1]) if basket else None}
