"""Generate tests/golden/ref_golden.npz from the reference's own CUDA code.

Runs on a B200 box: loads oracle/_ref/libmcqref.so (the reference's methods_cuda.cu built from
its sources by `make -C oracle ref`) and records
  * scrambled Sobol integers from the reference's curand Sobol32 + hh_scramble
    (methods_cuda.cu:781-819) for several salts / dimensions / offsets,
  * normals from its kernel_gen_hh_scrambled_sobol_normal (:799-825),
  * per-replica {sum Y, sum Y^2} of its accumulate_range steps (:1549-1622) with the point
    count pinned, for raw / Brownian-bridge / PCA noise and each model family,
  * results of its adaptive run_mc / run_mlmc / run_mlqmc drivers (statistical checks),
  * device time of the reference's pass for the RQMC Asian workload (the plain comparator).
Usage: python tests/golden/make_ref_golden.py [out.npz]

python tests/golden/make_ref_golden.py --levels writes ref_golden_levels.npz (+ .json) instead:
  * per-replica {sum dY, sum dY^2, sum Yf, sum Yf^2} of the reference's coupled level kernel
    kernel_mlmc (:445-518) as run_mlqmc_cuda runs a raw level (:1849-1919), GBM / Heston /
    Dupire, M = 2 and 4, levels 0-3 (golden_cases.level_cases),
  * per-replica {sum Y, sum Y^2} of its importance-sampling kernel kernel_is_gbm (:685-707) on
    scrambled Sobol normals (golden_cases.is_cases).
A case whose window holds a point with u = 1 (scrambled word >= 0xFFFFFF80) moves to the next
salt (+ 1000) until it has none; the JSON records the salt used.

python tests/golden/make_ref_golden.py --timing [N] prints the device time of the reference's own
pass for the RQMC Asian workload at 32 replicas x N points (default 2^20), raw and bridge.
"""
import ctypes as C
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)
import oracle_py as orc  # noqa: E402

T = orc.T
REF = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libmcqref.so"))
REF.mcqref_last_error.restype = C.c_char_p

from golden_cases import SALTS, OFFSETS, DIMS, cases as _cases, level_cases, is_cases  # noqa: E402


def ok(rc):
    if rc:
        raise RuntimeError(REF.mcqref_last_error().decode())


def ref_u32(salt, dim0, nd, off, n):
    out = np.zeros((nd, n), np.uint32)
    ok(REF.mcqref_sobol_u32(C.c_uint(salt), C.c_int(dim0), C.c_int(nd), C.c_uint(off), C.c_longlong(n),
                            out.ctypes.data_as(C.POINTER(C.c_uint))))
    return out


def ref_normal(salt, nd, off, n):
    out = np.zeros((nd, n), np.float32)
    ok(REF.mcqref_sobol_normal(C.c_uint(salt), C.c_int(nd), C.c_uint(off), C.c_longlong(n),
                               out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def ref_pass(m, p, n_steps, mode, salt0, R, off, N):
    sums = np.zeros(2 * R)
    ms = C.c_float()
    M = np.ascontiguousarray(orc.pca_matrix(n_steps, m.T).T.reshape(-1)) if mode == T.PCA else np.zeros(1)
    ok(REF.mcqref_qmc_pass(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_int(mode),
                           M.ctypes.data_as(C.POINTER(C.c_double)), C.c_uint(salt0), C.c_int(R), C.c_uint(off),
                           C.c_longlong(N), sums.ctypes.data_as(C.POINTER(C.c_double)), C.byref(ms)))
    return sums.reshape(R, 2), ms.value


def top_edge_hits(salt0, R, D, off, N):
    """Points whose scrambled integer maps to u == 1.0f (methods_cuda.cu:823) in the window."""
    hits = 0
    for r in range(R):
        for d0 in range(0, D, 64):
            nd = min(64, D - d0)
            hits += int((ref_u32(salt0 + r, d0, nd, off, N) >= 0xFFFFFF80).sum())
    return hits


def cases():
    return _cases(T)


def main(out):
    g = {}
    meta = {"cases": [], "drivers": {}, "timing": {}}
    for s in SALTS:
        for o in OFFSETS:
            for d0, nd in DIMS:
                g[f"u32_{s}_{o}_{d0}"] = ref_u32(s, d0, nd, o, 32)
    for o in (0, (1 << 22) - 1):
        g[f"normal_42_{o}"] = ref_normal(42, 16, o, 64)
    for name, m, p, n_steps, mode, salt0, R, off, N in cases():
        sums, _ = ref_pass(m, p, n_steps, mode, salt0, R, off, N)
        D = n_steps * T.noise_dim(m)
        hits = top_edge_hits(salt0, R, D, off, N)
        g["pass_" + name] = sums
        meta["cases"].append(dict(name=name, n_steps=n_steps, mode=mode, salt0=salt0, R=R, offset=off, N=N,
                                  top_edge_hits=hits))
        print(name, sums[:, 0] / N, "hits", hits, flush=True)
    # plain comparator: the reference's generate -> scale -> price steps for the RQMC Asian
    # workload (256 steps, 32 replicas) at 2^16 points per replica
    _, ms = ref_pass(T.gbm(100.0, 0.03, 0.25, 1.0), T.asian(100.0), 256, T.RAW, 42, 32, 0, 1 << 16)
    meta["timing"]["asian_raw_256_R32_N65536_ms"] = ms
    meta["timing"]["asian_raw_256_R32_N65536_path_steps_per_s"] = 32 * 65536 * 256 / (ms * 1e-3)
    _, ms = ref_pass(T.gbm(100.0, 0.03, 0.25, 1.0), T.asian(100.0), 256, T.BB, 42, 32, 0, 1 << 16)
    meta["timing"]["asian_bb_256_R32_N65536_ms"] = ms
    print("timing", meta["timing"], flush=True)
    # adaptive drivers (XORWOW inside, so statistical comparisons only)
    o4 = np.zeros(4)
    pd = o4.ctypes.data_as(C.POINTER(C.c_double))
    gbm, eur = T.gbm(100.0, 0.05, 0.2, 1.0), T.european(100.0, 0.05, 1.0)
    t0 = time.time()
    ok(REF.mcqref_run_mc(C.byref(gbm), C.byref(eur), C.c_double(1e-2), 64, pd))
    meta["drivers"]["mc_gbm_eur_64_eps1e-2"] = list(o4) + [time.time() - t0]
    ok(REF.mcqref_run_mlmc(C.byref(gbm), C.byref(eur), C.c_double(1e-2), 2, 10, 400, pd))
    meta["drivers"]["mlmc_gbm_eur_eps1e-2"] = list(o4)
    hes = T.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    ok(REF.mcqref_run_mlqmc(C.byref(hes), C.byref(T.european(100.0, 0.02, 1.0)), C.c_double(1e-2), 4, 8, 400, 16,
                            pd))
    meta["drivers"]["mlqmc_heston_eur_M4_eps1e-2"] = list(o4)
    ok(REF.mcqref_run_mlqmc(C.byref(gbm), C.byref(eur), C.c_double(5e-3), 2, 10, 400, 16, pd))
    meta["drivers"]["mlqmc_gbm_eur_eps5e-3"] = list(o4)
    print("drivers", meta["drivers"], flush=True)
    np.savez_compressed(out, **g)
    with open(os.path.splitext(out)[0] + ".json", "w") as f:
        json.dump(meta, f, indent=1)


def ref_level(m, p, level, M, salt0, R, off, N):
    sums = np.zeros(4 * R)
    n_fine = M ** level
    ok(REF.mcqref_level_pass(C.byref(m), C.byref(p), C.c_int(n_fine), C.c_int(M), C.c_int(int(level == 0)),
                             C.c_uint(salt0), C.c_int(R), C.c_uint(off), C.c_longlong(N),
                             sums.ctypes.data_as(C.POINTER(C.c_double))))
    return sums.reshape(R, 4)


def ref_is(m, p, n_steps, z_step, salt0, R, off, N):
    sums = np.zeros(2 * R)
    ok(REF.mcqref_is_pass(C.byref(m), C.byref(p), C.c_int(n_steps), C.c_double(z_step), C.c_uint(salt0),
                          C.c_int(R), C.c_uint(off), C.c_longlong(N), sums.ctypes.data_as(C.POINTER(C.c_double))))
    return sums.reshape(R, 2)


def main_levels(out):
    g, meta = {}, {"levels": [], "is": []}
    for name, m, p, level, M, salt0, R, off, N in level_cases(T):
        D = M ** level * T.noise_dim(m)
        while top_edge_hits(salt0, R, D, off, N):
            salt0 += 1000
        g[name] = ref_level(m, p, level, M, salt0, R, off, N)
        meta["levels"].append(dict(name=name, level=level, M=M, salt0=salt0, R=R, offset=off, N=N))
        print(name, salt0, g[name][:, 0] / N, g[name][:, 2] / N, flush=True)
    for name, m, p, n_steps, z_star, salt0, R, off, N in is_cases(T):
        while top_edge_hits(salt0, R, n_steps, off, N):
            salt0 += 1000
        z_step = z_star / np.sqrt(n_steps)
        g[name] = ref_is(m, p, n_steps, z_step, salt0, R, off, N)
        meta["is"].append(dict(name=name, n_steps=n_steps, z_star=z_star, z_step=z_step, salt0=salt0, R=R,
                               offset=off, N=N))
        print(name, salt0, g[name][:, 0] / N, flush=True)
    np.savez_compressed(out, **g)
    with open(os.path.splitext(out)[0] + ".json", "w") as f:
        json.dump(meta, f, indent=1)


def main_timing(n_per_replica):
    """Device time of the reference's own generate -> transform -> price steps for the RQMC Asian
    workload (GBM, 256 steps, 32 replicas x n_per_replica points), raw and Brownian-bridge
    ordering, after one warm-up pass each: the GPU path the engine's fused pass replaces."""
    m, p = T.gbm(100.0, 0.03, 0.25, 1.0), T.asian(100.0)
    out = {}
    for name, mode in (("raw", T.RAW), ("bridge", T.BB)):
        ref_pass(m, p, 256, mode, 42, 1, 0, 1 << 14)
        sums, ms = ref_pass(m, p, 256, mode, 42, 32, 0, n_per_replica)
        out[name] = {"ms": ms, "path_steps_per_s": 32 * n_per_replica * 256 / (ms * 1e-3),
                     "price": float((sums[:, 0] / n_per_replica).mean())}
    print(json.dumps({"reference_gpu_asian_256_R32": dict(out, points_per_replica=n_per_replica)}))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--timing":
        main_timing(int(sys.argv[2]) if len(sys.argv) > 2 else 1 << 20)
    elif len(sys.argv) > 1 and sys.argv[1] == "--levels":
        main_levels(os.path.join(HERE, "ref_golden_levels.npz"))
    else:
        main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_golden.npz"))
