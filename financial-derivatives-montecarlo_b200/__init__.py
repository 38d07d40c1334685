"""Python binding of the B200 pricing engine (libmcq.so) through its C ABI (include/mcq.h).

The engine itself is C++/CUDA; this module only marshals arguments.  Importing it loads the
in-tree libmcq.so and raises if the library is missing — there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

from . import mcq_types as T
from .mcq_types import (  # noqa: F401  (re-exported builders)
    GBM, HESTON, DUPIRE, MULTI_DUPIRE, LOCALVOL_GRID, BASKET_GBM,
    EUROPEAN, ASIAN, GEOM_ASIAN, LOOKBACK, BARRIER_UP_OUT, BASKET, BARRIER_DOWN_OUT,
    RAW, BB, PCA, FLAG_COMPAT_U_INF, FLAG_COMPAT_HESTON_MLMC, FLAG_HESTON_MILSTEIN, FLAG_BASKET_OWN_S0,
    BOOK_BATCHED, BOOK_PLAIN, book_option, book_single, mixed_singles, config5_book,
    gbm, heston, dupire, multi_dupire, basket_gbm, localvol_grid, config4_surface, payoff, european, asian,
    geom_asian, lookback, barrier_up_out, barrier_down_out, basket, noise_dim,
)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmcq.so")

EXPORTS = [
    "mcq_init", "mcq_shutdown", "mcq_last_error", "mcq_version", "mcq_default_cfgs", "mcq_model_heston",
    "mcq_bb_create", "mcq_pca_create", "mcq_pca_create_from", "mcq_handle_free", "mcq_handle_info",
    "mcq_run_mc", "mcq_run_mc_fixed", "mcq_run_qmc", "mcq_run_mlmc", "mcq_run_mlqmc", "mcq_cv_pilot",
    "mcq_run_mc_cv", "mcq_run_qmc_cv", "mcq_run_is", "mcq_qmc_pass", "mcq_qmc_pass_device",
    "mcq_mc_pass", "mcq_level_pass", "mcq_is_pass", "mcq_sobol_hh_u32", "mcq_sobol_hh_normal", "mcq_philox4x32_10",
    "mcq_bb_tables", "mcq_pca_matrix", "mcq_debug_pass_dump", "mcq_debug_wait_timeout",
    "mcq_debug_last_pass_layout", "mcq_qmc_pass_noalloc", "mcq_adjoint",
    "mcq_book_price", "mcq_book_level_sums", "mcq_book_create", "mcq_book_submit", "mcq_book_size",
    "mcq_book_run", "mcq_book_clear", "mcq_book_free",
]


class MCQError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mcq error {code}: {msg}")
        self.code = code


_lib = None
_P = C.POINTER


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run financial-derivatives-montecarlo_b200/build.py")
        L = C.CDLL(LIB_PATH)
        L.mcq_last_error.restype = C.c_char_p
        for name in EXPORTS:
            if name != "mcq_last_error":
                getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise MCQError(rc, lib().mcq_last_error().decode())


def init(device=-1):
    _check(lib().mcq_init(C.c_int(device)))


def shutdown():
    _check(lib().mcq_shutdown())


def version():
    return lib().mcq_version()


def mc_cfg(**kw):
    c = T.MCCfg()
    lib().mcq_default_cfgs(C.byref(c), None, None)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def qmc_cfg(**kw):
    c = T.QMCCfg()
    lib().mcq_default_cfgs(None, C.byref(c), None)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def mlmc_cfg(**kw):
    c = T.MLMCCfg()
    lib().mcq_default_cfgs(None, None, C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class Handle:
    """BB / PCA handle (DeviceBBData / DevicePCAData); freed on close() or garbage collection."""

    def __init__(self, ptr, kind, n):
        self.ptr, self.kind, self.n = ptr, kind, n

    def close(self):
        if self.ptr:
            lib().mcq_handle_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bb_create(N, T_):
    h = C.c_void_p()
    _check(lib().mcq_bb_create(C.c_int(N), C.c_double(T_), C.byref(h)))
    return Handle(h, BB, N)


def pca_create(m, T_):
    h = C.c_void_p()
    _check(lib().mcq_pca_create(C.c_int(m), C.c_double(T_), C.byref(h)))
    return Handle(h, PCA, m)


def _h(x):
    return x.ptr if x is not None else None


def bb_tables(h):
    n = h.n
    mi = np.zeros(n, np.int32)
    wl, wr, sd = (np.zeros(n, np.float32) for _ in range(3))
    _check(lib().mcq_bb_tables(_h(h), mi.ctypes.data_as(_P(C.c_int)), wl.ctypes.data_as(_P(C.c_float)),
                               wr.ctypes.data_as(_P(C.c_float)), sd.ctypes.data_as(_P(C.c_float))))
    return mi, wl, wr, sd


def pca_matrix(h):
    M = np.zeros(h.n * h.n, np.float32)
    _check(lib().mcq_pca_matrix(_h(h), M.ctypes.data_as(_P(C.c_float))))
    return M.reshape(h.n, h.n).T  # M[i, k]


def _res():
    return T.Result()


def run_mc(m, p, eps, n_steps, cfg=None):
    r = _res()
    _check(lib().mcq_run_mc(C.byref(m), C.byref(p), C.c_double(eps), C.c_int(n_steps),
                            C.byref(cfg or mc_cfg()), C.byref(r)))
    return r.as_dict()


def run_mc_fixed(m, p, n_steps, n_paths, seed):
    a, b = C.c_double(), C.c_double()
    _check(lib().mcq_run_mc_fixed(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_int64(n_paths),
                                  C.c_uint32(seed), C.byref(a), C.byref(b)))
    return a.value, b.value


def run_qmc(m, p, eps, n_steps, cfg=None, noise=RAW, bb=None, pca=None):
    r = _res()
    _check(lib().mcq_run_qmc(C.byref(m), C.byref(p), C.c_double(eps), C.c_int(n_steps),
                             C.byref(cfg or qmc_cfg()), C.c_int(noise), _h(bb), _h(pca), C.byref(r)))
    return r.as_dict()


def run_mlmc(m, p, eps, cfg=None):
    r = _res()
    _check(lib().mcq_run_mlmc(C.byref(m), C.byref(p), C.c_double(eps), C.byref(cfg or mlmc_cfg()), C.byref(r)))
    return r.as_dict()


def run_mlqmc(m, p, eps, ml=None, qc=None, noise=RAW, bb_list=(), pca_list=()):
    r = _res()
    nb, npc = len(bb_list), len(pca_list)
    bl = (C.c_void_p * max(nb, 1))(*[_h(b) for b in bb_list])
    pl = (C.c_void_p * max(npc, 1))(*[_h(b) for b in pca_list])
    _check(lib().mcq_run_mlqmc(C.byref(m), C.byref(p), C.c_double(eps), C.byref(ml or mlmc_cfg()),
                               C.byref(qc or qmc_cfg()), C.c_int(noise), bl, C.c_int(nb), pl, C.c_int(npc),
                               C.byref(r)))
    return r.as_dict()


def cv_pilot(main_m, ctrl_m, main_p, ctrl_p, E_ctrl, n_steps, N_pilot, seed=0):
    o = T.CVPilotOut()
    _check(lib().mcq_cv_pilot(C.byref(main_m), C.byref(ctrl_m), C.byref(main_p), C.byref(ctrl_p),
                              C.c_double(E_ctrl), C.c_int(n_steps), C.c_int(N_pilot), C.c_uint32(seed), C.byref(o)))
    return {"beta": o.beta, "var_plain": o.var_plain, "var_cv": o.var_cv}


def run_mc_cv(main_m, ctrl_m, main_p, ctrl_p, E_ctrl, beta, eps, n_steps, cfg=None):
    r = _res()
    _check(lib().mcq_run_mc_cv(C.byref(main_m), C.byref(ctrl_m), C.byref(main_p), C.byref(ctrl_p),
                               C.c_double(E_ctrl), C.c_double(beta), C.c_double(eps), C.c_int(n_steps),
                               C.byref(cfg or mc_cfg()), C.byref(r)))
    return r.as_dict()


def run_qmc_cv(main_m, ctrl_m, main_p, ctrl_p, E_ctrl, beta, eps, n_steps, cfg=None):
    r = _res()
    _check(lib().mcq_run_qmc_cv(C.byref(main_m), C.byref(ctrl_m), C.byref(main_p), C.byref(ctrl_p),
                                C.c_double(E_ctrl), C.c_double(beta), C.c_double(eps), C.c_int(n_steps),
                                C.byref(cfg or qmc_cfg()), C.byref(r)))
    return r.as_dict()


def run_is(m, p, z_star, eps, cfg=None):
    r = _res()
    _check(lib().mcq_run_is(C.byref(m), C.byref(p), C.c_double(z_star), C.c_double(eps),
                            C.byref(cfg or mc_cfg()), C.byref(r)))
    return r.as_dict()


def qmc_pass(m, p, n_steps, noise=RAW, bb=None, pca=None, salt_base=42, R=1, offset=0, n_points=1024, flags=0):
    out = np.zeros((R, 2), np.float64)
    _check(lib().mcq_qmc_pass(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_int(noise), _h(bb), _h(pca),
                              C.c_uint32(salt_base), C.c_int(R), C.c_uint32(offset), C.c_int64(n_points),
                              C.c_int(flags), out.ctypes.data_as(_P(C.c_double))))
    return out


def qmc_pass_device(m, p, n_steps, sums_device_ptr, stream_ptr=0, noise=RAW, bb=None, pca=None, salt_base=42,
                    R=1, offset=0, n_points=1024, flags=0):
    _check(lib().mcq_qmc_pass_device(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_int(noise), _h(bb), _h(pca),
                                     C.c_uint32(salt_base), C.c_int(R), C.c_uint32(offset), C.c_int64(n_points),
                                     C.c_int(flags), C.c_void_p(sums_device_ptr), C.c_void_p(stream_ptr)))


def qmc_pass_noalloc(m, p, n_steps, sums_device_ptr, stream_ptr=0, salt_base=42, R=1, offset=0, n_points=1024,
                     flags=0):
    """mcq_qmc_pass_noalloc: the RQMC pass with all scratch in the library's fixed device array."""
    _check(lib().mcq_qmc_pass_noalloc(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_uint32(salt_base), C.c_int(R),
                                      C.c_uint32(offset), C.c_int64(n_points), C.c_int(flags),
                                      C.c_void_p(sums_device_ptr), C.c_void_p(stream_ptr)))


def adjoint(m, p, n_steps, salt_base=42, R=16, offset=0, n_points=4096, flags=0):
    """mcq_adjoint: pathwise Greeks; returns (dict, node_vega array or None)."""
    g = T.Greeks()
    nodes = np.zeros(m.lv_nK * m.lv_nt, np.float64) if m.kind == LOCALVOL_GRID else None
    _check(lib().mcq_adjoint(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_uint32(salt_base), C.c_int(R),
                             C.c_uint32(offset), C.c_int64(n_points), C.c_int(flags), C.byref(g),
                             nodes.ctypes.data_as(_P(C.c_double)) if nodes is not None else None))
    d = {k: getattr(g, k) for k, _ in g._fields_}
    if nodes is not None:
        nodes = nodes.reshape(m.lv_nt, m.lv_nK)
    return d, nodes


def book_price(options, mode=BOOK_BATCHED, ml=None, qc=None):
    """mcq_book_price: MLQMC price and per-asset pathwise delta of every option of a book.
    Returns (list of dicts {price, std_error, delta (n_assets,), n_samples, levels, converged},
    stats dict).  ml / qc default to M = 2, pilot_n = 400, n0_steps = 1 and R = 16, salt 42."""
    n = len(options)
    arr = (T.BookOption * n)(*options)
    out = (T.BookResult * n)()
    st = T.BookStats()
    ml = ml if ml is not None else mlmc_cfg(M=2, n0_steps=1)
    qc = qc if qc is not None else qmc_cfg(R=16)
    _check(lib().mcq_book_price(arr, C.c_int(n), C.byref(ml), C.byref(qc), C.c_int(mode), out, C.byref(st)))
    res = []
    for o, r in zip(options, out):
        res.append({"price": r.price, "std_error": r.std_error, "delta": np.array(r.delta[:o.n_assets]),
                    "n_samples": r.n_samples, "levels": r.levels, "converged": bool(r.converged)})
    return res, st.as_dict()


class Book:
    """mcq_book: a book built up by submit() and priced by run() (the same pricing as book_price).
    The library copies the submitted options, so the Python option objects may be dropped."""

    def __init__(self):
        self.h = C.c_void_p()
        _check(lib().mcq_book_create(C.byref(self.h)))

    def submit(self, options):
        arr = (T.BookOption * len(options))(*options)
        _check(lib().mcq_book_submit(self.h, arr, C.c_int(len(options))))

    def __len__(self):
        n = C.c_int()
        _check(lib().mcq_book_size(self.h, C.byref(n)))
        return n.value

    def run(self, mode=BOOK_BATCHED, ml=None, qc=None):
        n = len(self)
        out = (T.BookResult * n)()
        st = T.BookStats()
        ml = ml if ml is not None else mlmc_cfg(M=2, n0_steps=1)
        qc = qc if qc is not None else qmc_cfg(R=16)
        _check(lib().mcq_book_run(self.h, C.byref(ml), C.byref(qc), C.c_int(mode), out, C.byref(st)))
        return out, st.as_dict()

    def clear(self):
        _check(lib().mcq_book_clear(self.h))

    def close(self):
        if self.h:
            _check(lib().mcq_book_free(self.h))
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def book_level_sums(option, level, offset=0, n_points=1024, ml=None, qc=None):
    """mcq_book_level_sums: [R][4 + n_assets] sums of one slice, through the book kernel."""
    ml = ml if ml is not None else mlmc_cfg(M=2, n0_steps=1)
    qc = qc if qc is not None else qmc_cfg(R=16)
    out = np.zeros((qc.R, 20), np.float64)
    _check(lib().mcq_book_level_sums(C.byref(option), C.byref(ml), C.byref(qc), C.c_int(level), C.c_uint32(offset),
                                     C.c_int64(n_points), out.ctypes.data_as(_P(C.c_double))))
    return out[:, :4 + option.n_assets]


def debug_wait_timeout(polls=1000):
    """mcq_debug_wait_timeout: a bounded device wait that is made to give up (raises MCQError 7)."""
    _check(lib().mcq_debug_wait_timeout(C.c_uint32(polls)))


def mc_pass(m, p, n_steps, seed, stream_id, first_path, n_paths):
    out = np.zeros(2, np.float64)
    _check(lib().mcq_mc_pass(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_uint32(seed), C.c_uint32(stream_id),
                             C.c_int64(first_path), C.c_int64(n_paths), out.ctypes.data_as(_P(C.c_double))))
    return out


def level_pass(m, p, n_fine, M, noise=RAW, bb=None, pca=None, use_sobol=True, seed=42, salt_base=42, R=1,
               offset=0, n_points=1024, flags=0):
    """M <= 0 means level 0 (no coarse path)."""
    out = np.zeros((R, 4), np.float64)
    _check(lib().mcq_level_pass(C.byref(m), C.byref(p), C.c_int(n_fine), C.c_int(M), C.c_int(noise), _h(bb),
                                _h(pca), C.c_int(int(use_sobol)), C.c_uint32(seed), C.c_uint32(salt_base),
                                C.c_int(R), C.c_uint32(offset), C.c_int64(n_points), C.c_int(flags),
                                out.ctypes.data_as(_P(C.c_double))))
    return out


def is_pass(m, p, n_steps, z_star_step, use_sobol=True, seed=42, salt_base=42, R=1, offset=0, n_points=1024,
            flags=0):
    """Importance-sampling pass (kernel_is_gbm): [R][2] {sum Y, sum Y^2}; z_star_step per step."""
    out = np.zeros((R, 2), np.float64)
    _check(lib().mcq_is_pass(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_double(z_star_step),
                             C.c_int(int(use_sobol)), C.c_uint32(seed), C.c_uint32(salt_base), C.c_int(R),
                             C.c_uint32(offset), C.c_int64(n_points), C.c_int(flags),
                             out.ctypes.data_as(_P(C.c_double))))
    return out


def debug_pass_dump(m, n_steps, noise=RAW, bb=None, use_sobol=True, seed=0, salt_base=42, R=1, offset=0,
                    n_points=32, flags=0):
    D = n_steps * noise_dim(m)
    out = np.zeros((R, n_points, D), np.float32)
    _check(lib().mcq_debug_pass_dump(C.byref(m), C.c_int(n_steps), C.c_int(noise), _h(bb), C.c_int(int(use_sobol)),
                                     C.c_uint32(seed), C.c_uint32(salt_base), C.c_int(R), C.c_uint32(offset),
                                     C.c_int64(n_points), C.c_int(flags), out.ctypes.data_as(_P(C.c_float))))
    return out


def debug_last_pass_layout():
    """(groups per work item, carried Sobol start words per warp) of the last fused pass."""
    g, c = C.c_int(0), C.c_int(0)
    _check(lib().mcq_debug_last_pass_layout(C.byref(g), C.byref(c)))
    return g.value, c.value


def sobol_hh_u32(salt, dim0, nd, offset, n):
    out = np.zeros((nd, n), np.uint32)
    _check(lib().mcq_sobol_hh_u32(C.c_uint32(salt), C.c_int(dim0), C.c_int(nd), C.c_uint32(offset),
                                  C.c_int64(n), out.ctypes.data_as(_P(C.c_uint32))))
    return out


def sobol_hh_normal(salt, dim0, nd, offset, n, flags=0):
    out = np.zeros((nd, n), np.float32)
    _check(lib().mcq_sobol_hh_normal(C.c_uint32(salt), C.c_int(dim0), C.c_int(nd), C.c_uint32(offset),
                                     C.c_int64(n), C.c_int(flags), out.ctypes.data_as(_P(C.c_float))))
    return out


def philox(ctr, key):
    o = (C.c_uint32 * 4)()
    _check(lib().mcq_philox4x32_10((C.c_uint32 * 4)(*ctr), (C.c_uint32 * 2)(*key), o))
    return list(o)
