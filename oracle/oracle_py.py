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


def path_payoff(m, p, n_steps, z, nz=None):
    z = np.ascontiguousarray(z, dtype=np.float64)
    return lib().orc_path_payoff(C.byref(m), C.byref(p), C.c_int(n_steps), C.byref(nz) if nz else None,
                                 z.ctypes.data_as(_pd))


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


def basket_level(m, p, n_fine, M, z):
    """One coupled basket path pair: (Yf, Yc, dd[n_assets]); M <= 0 is level 0."""
    z = np.ascontiguousarray(z, dtype=np.float64)
    dd = np.zeros(m.n_assets)
    yc = C.c_double()
    L = lib()
    L.orc_basket_level.restype = C.c_double
    yf = L.orc_basket_level(C.byref(m), C.byref(p), C.c_int(n_fine), C.c_int(M), z.ctypes.data_as(_pd),
                            C.byref(yc), dd.ctypes.data_as(_pd))
    return yf, yc.value, dd


def basket_level_sums(m, p, n_fine, M, salt_base=42, R=1, offset=0, N=1024, flags=0, threads=0):
    out = np.zeros((R, 4 + m.n_assets))
    rc = lib().orc_basket_level_sums(C.byref(m), C.byref(p), C.c_int(n_fine), C.c_int(M), C.c_uint32(salt_base),
                                     C.c_int(R), C.c_uint32(offset), C.c_int64(N), C.c_int(flags), C.c_int(threads),
                                     out.ctypes.data_as(_pd))
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
