#!/usr/bin/env python
"""Benchmark of the fused RQMC path kernel on the reference's headline workload.

Workload (the RQMC configuration the metric is quoted on): arithmetic-average Asian call under
GBM, S0 = K = 100, r = mu = 0.03, sigma = 0.25, T = 1, 256 Euler steps = 256 Hong–Hickernell
scrambled Sobol dimensions, R = 32 replicas with salts 42.., raw noise ordering.

  value  one "step" = one fused pass over 32 replicas x N points x 256 steps (default
         N = 2^20 per replica, 8.6e9 path-steps), inputs (direction tables, parameters)
         resident, sums left on the device; device time from CUDA events on the launching
         stream; L2 flushed (256 MiB write) between steps.
  e2e    the reference-facing driver call mcq_run_qmc (run_qmc_cuda's entry point) at
         eps = 1e-3 from 2^14 points per replica, doubling until var_of_means < eps^2/2, with
         host structs in and the result read back; path-steps of the whole adaptive run over
         host wall time.
Multi-GPU (torchrun): one estimator of 32 N replicas split in blocks of 32 over the N ranks
(rank k owns the replicas of salts 42 + 32 k ..), the only exchange the estimator has: after each
pass one all-reduce of the [32 N][2] FP64 per-replica sums (every slot with one contributor, so
the reduced sums are the one-process sums bit for bit) gives every rank the estimator; max over
ranks of the device time; "scaling": "weak".  The e2e leg at N > 1 runs the same split through
the adaptive doubling loop (sharded.run_qmc_sharded over mcq_qmc_pass, one all-reduce per
doubling) with R = 32 N.
--impl reference times the reference algorithm's CPU restatement (the oracle) on the host
cores on a bounded sample of the same workload (the reference has no CPU path of its own).
"""
import argparse
import importlib.util
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "financial-derivatives-montecarlo_b200")

S0, K, R_, SIG, T_, STEPS, REPS, SALT = 100.0, 100.0, 0.03, 0.25, 1.0, 256, 32, 42
METRIC = "path-steps/s"
# Algorithmic FP32 work per path-step of the raw Sobol GBM Asian path, counted as written in the
# reference (each +, -, x, /, min, max one flop; special functions apart): the scrambled-Sobol
# normal's u = (x + 1) 2^-32 (2 flops) and one inverse normal (an SFU-class call, not counted as
# flops), the GBM step S + mu S h + sigma S sqrt(h) z with the sqrt(h) scale (7 flops,
# methods_cuda.cu:273), the Kahan-compensated running sum of the Asian average (4 flops).
FLOPS_PER_PATH_STEP = 2 + 7 + 4
SFU_PER_PATH_STEP = 1
# The same path-step with the inverse normal counted as the AS241 central rational it evaluates
# (7 + 7 FMA + 1 division: 29 flops): an issue model, not the algorithmic count.
ISSUE_MODEL_FLOPS_PER_PATH_STEP = 2 + 29 + 4 + 4


def load_engine():
    spec = importlib.util.spec_from_file_location("fdmc_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["fdmc_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def wait_rows(self, n, timeout):
        """Wait (at most `timeout` s) until at least n samples have arrived; nvidia-smi takes a
        while to start, longer than a short timed region."""
        t0 = time.time()
        while self.proc and len(self.rows) < n and time.time() - t0 < timeout:
            time.sleep(0.01)

    def summary(self, first=0):
        rows = self.rows[first:]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max((float(r[2]) for r in rows if r[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def oracle_values():
    """FP64 oracle values of the benchmark's workloads (tests/golden/oracle_values.json, written by
    tests/golden/make_oracle_values.py: closed forms where they exist, FP64 oracle runs otherwise)."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "oracle_values.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def vs_oracle(price, se, ref, ref_se=0.0, kind=""):
    """A result's error against an FP64 oracle value, in absolute terms and in standard errors of
    the difference."""
    if ref is None:
        return None
    comb = math.hypot(se or 0.0, ref_se or 0.0)
    return {"oracle": ref, "oracle_se": ref_se, "error": price - ref, "combined_se": comb,
            "error_in_se": (price - ref) / comb if comb > 0 else None, "oracle_kind": kind}


def bs_call(S0, K, T, r, sigma):
    """Black–Scholes call in FP64 (the closed form the one-asset book options are checked against)."""
    if T <= 0 or sigma <= 0:
        return max(S0 - K * math.exp(-r * T), 0.0)
    d1 = (math.log(S0 / K) + (r + 0.5 * sigma * sigma) * T) / (sigma * math.sqrt(T))
    d2 = d1 - sigma * math.sqrt(T)
    N = lambda x: 0.5 * math.erfc(-x / math.sqrt(2.0))   # noqa: E731
    return S0 * N(d1) - K * math.exp(-r * T) * N(d2)


def cpu_baseline(seconds=12.0, steps=1):
    """Oracle (CPU restatement, FP64 paths) on all host threads: returns path-steps/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as orc
    T = orc.T
    m, p = T.gbm(S0, R_, SIG, T_), T.asian(K)
    threads = orc.max_threads()
    # size the sample to about `seconds` of wall time from a short calibration run
    n = 256
    t0 = time.perf_counter()
    orc.qmc_sums(m, p, STEPS, None, SALT, REPS, 0, n, 0, threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    n = max(256, int(n * seconds / dt) // 256 * 256)
    vals = []
    for _ in range(steps):
        t0 = time.perf_counter()
        orc.qmc_sums(m, p, STEPS, None, SALT, REPS, 0, n, 0, threads)
        dt = time.perf_counter() - t0
        vals.append(REPS * n * STEPS / dt)
    v = sorted(vals)[len(vals) // 2]
    return {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{REPS} replicas x {n} points x {STEPS} steps of the same workload (FP64 oracle)"}


def configs_bench(eng, orv):
    """The other workloads of the benchmark suite through the public API, host wall time of one
    warm call each, each result stated against its FP64 oracle value: plain MC (GBM European, 64
    Euler steps, Philox, pilot 2^14, eps 1e-2; Black–Scholes), MLQMC for Heston with the
    Euler-Milstein full-truncation variance step (kappa 2, theta 0.04, xi 0.3, rho -0.7, v0 0.04,
    S0 100, r 0.02, T 1; M 4, 4 steps on level 0, L <= 8, R 16, eps 1e-3) with a lookback and a
    down-and-out call (K 100, B 80; FP64 oracle MLQMC at eps 5e-4), and the pathwise adjoint on
    the 64 x 32 local-vol grid (Asian call, T 2, 512 steps, 16 x 2^18 scrambled paths, price +
    delta + rho + 2048 node vegas; FP64 oracle price and central differences)."""
    out = {}

    def timed(fn):
        fn()
        t0 = time.perf_counter()
        r = fn()
        return r, time.perf_counter() - t0

    m, p = eng.gbm(100.0, 0.05, 0.2, 1.0), eng.european(100.0, 0.05, 1.0)
    r, t = timed(lambda: eng.run_mc(m, p, 1e-2, 64, eng.mc_cfg(pilot_n=1 << 14)))
    o = orv.get("mc_gbm_european", {})
    out["mc_gbm_european"] = {"price": r["price"], "std_error": r["std_error"], "time_s": t,
                              "path_steps_per_s": r["path_steps"] / t,
                              "vs_oracle": vs_oracle(r["price"], r["std_error"], o.get("value"), 0.0, o.get("kind", ""))}
    h = eng.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
    for name, pay in (("lookback", eng.lookback(0.2)), ("down_out", eng.barrier_down_out(100.0, 80.0, 0.2, 0.02, 1.0))):
        r, t = timed(lambda: eng.run_mlqmc(h, pay, 1e-3, eng.mlmc_cfg(M=4, n0_steps=4, max_L=8,
                                                                     flags=eng.FLAG_HESTON_MILSTEIN),
                                           eng.qmc_cfg(R=16)))
        o = orv.get("mlqmc_heston_" + name, {})
        out["mlqmc_heston_" + name] = {"price": r["price"], "std_error": r["std_error"], "levels": r["levels"],
                                       "converged": bool(r["converged"]), "time_s": t,
                                       "path_steps_per_s": r["path_steps"] / t,
                                       "vs_oracle": vs_oracle(r["price"], r["std_error"], o.get("value"), o.get("se", 0.0),
                                                              o.get("kind", ""))}
    K, tt, grid = eng.config4_surface()
    lv = eng.localvol_grid(K, tt, grid, 100.0, 0.05, 2.0)
    (g, _), t = timed(lambda: eng.adjoint(lv, eng.asian(100.0), 512, salt_base=42, R=16, n_points=1 << 18))
    o = orv.get("adjoint_localvol_asian", {})
    greeks = {}
    for k in ("delta", "rho", "vega"):
        if k in o:
            greeks[k] = {"oracle_fd": o[k], "error": g[k] - o[k], "rel_error": (g[k] - o[k]) / abs(o[k])}
    out["adjoint_localvol_asian"] = {"price": g["price"], "price_se": g["price_se"], "delta": g["delta"], "rho": g["rho"],
                                     "vega": g["vega"], "time_s": t, "path_steps_per_s": g["path_steps"] / t,
                                     "paths_per_s": g["n_paths"] / t,
                                     "vs_oracle": vs_oracle(g["price"], g["price_se"], o.get("price"),
                                                            o.get("price_se", 0.0), o.get("kind", "")),
                                     "greeks_vs_oracle_fd": greeks or None}
    return out


def book_checks(eng, opts, res, orv, first_index=0):
    """Convergence counts and FP64-oracle errors of one book run: options whose bias test passed,
    options whose standard error reached their eps, one-asset options against Black–Scholes (their
    basket is the asset itself), and the sampled multi-asset options against the FP64 oracle's
    MLQMC values."""
    import numpy as np
    conv = sum(1 for x in res if x["converged"])
    se_ok = sum(1 for o, x in zip(opts, res) if x["std_error"] <= o.eps)
    one = []
    for o, x in zip(opts, res):
        if not o.model and o.n_assets == 1:
            ref = bs_call(float(o.S0[0]), o.K, o.T, o.r, float(o.sigma[0]))
            one.append((x["price"] - ref, x["std_error"], o.eps, x["converged"]))
    out = {"options": len(opts), "converged": conv, "se_le_eps": se_ok}
    if one:
        e = np.array([a for a, _, _, _ in one])
        z = np.array([abs(a) / b if b > 0 else 0.0 for a, b, _, _ in one])
        conv1 = [(a, b, ep) for a, b, ep, c in one if c]
        ok = sum(1 for a, b, ep in conv1 if abs(a) <= ep / math.sqrt(2.0) + 3 * b)
        out["one_asset_vs_black_scholes"] = {
            "n": len(one), "max_abs_error": float(np.abs(e).max()), "mean_abs_error": float(np.abs(e).mean()),
            "median_abs_error_in_se": float(np.median(z)),
            "converged": len(conv1), "converged_within_bias_bound_plus_3se": ok,
            "note": "error = MLQMC price - Black-Scholes; the MLQMC estimate targets the finest level's Euler "
                    "price, whose bias the stopping test bounds by eps/sqrt(2) when the option converged"}
    samp = orv.get("book", {}).get("options", {})
    rows = []
    for k, v in samp.items():
        i = int(k) - first_index
        if 0 <= i < len(res):
            rows.append({"option": int(k), "assets": v.get("assets"),
                         **vs_oracle(res[i]["price"], res[i]["std_error"], v["value"], v.get("se", 0.0),
                                     orv["book"].get("kind", ""))})
    if rows:
        out["sample_vs_fp64_oracle"] = rows
    return out


def book_bench(eng, n, n_loose, orv, n_all=0):
    """The batched heterogeneous book against its plain form on the same GPU: the first n options
    of the 4096-option synthetic book (d ~ U{1..16}, correlated GBM, Dirichlet weights, T ~
    U[0.1, 3], 16-512 finest steps, eps ~ U[5e-4, 5e-3]), each priced by MLQMC (R = 16, M = 2)
    with its per-asset pathwise deltas: at each option's own eps, at the metric's eps = 1e-3 for
    every option, and (the first n_loose options) at the loosest eps of the range, 5e-3; the first
    n_all options at eps = 1e-3 in the batched form only (the full-size configuration).  Each mode
    is timed by the library around its pricing loop (host wall time with the device
    synchronised), after a warm-up book.  Under torchrun the options are dealt round-robin over the
    ranks (the same n in total) and the time is the maximum over ranks."""
    import torch
    rank, _, world = dist_env()
    book = eng.config5_book(n=4096, seed=5)
    # warm-up: one option of every basket width (all kernels loaded, graphs and streams set up)
    warm = []
    for d in range(1, 17):
        o = next(o for o in book if o.n_assets == d)
        c = type(o).from_buffer_copy(o)   # same arrays (kept alive by `book`), coarser target
        c.eps = 20 * o.eps
        warm.append(c)
    eng.book_price(warm, eng.BOOK_BATCHED)
    eng.book_price(warm, eng.BOOK_PLAIN)

    def both_modes(opts, total):
        d, res = {}, {}
        for name, mode in (("batched", eng.BOOK_BATCHED), ("plain", eng.BOOK_PLAIN)):
            r, st = eng.book_price(opts, mode) if opts else ([], {"time_s": 0.0, "rounds": 0, "launches": 0,
                                                                  "normals": 0.0, "path_steps": 0.0})
            res[name] = r
            agg = torch.tensor([st["time_s"], st["normals"], st["path_steps"]], dtype=torch.float64, device="cuda")
            if world > 1:
                t = agg[:1].clone()
                torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
                w = agg[1:].clone()
                torch.distributed.all_reduce(w, op=torch.distributed.ReduceOp.SUM)
                agg = torch.cat([t, w])
            tmax, normals, psteps = agg.tolist()
            d[name] = {"options_per_s": total / tmax, "time_s": tmax, "rounds": st["rounds"],
                       "launches": st["launches"], "normals_per_s": normals / tmax,
                       "path_steps_per_s": psteps / tmax}
        d["batched_over_plain"] = d["batched"]["options_per_s"] / d["plain"]["options_per_s"]
        same = lambda x, y: x == y or (x != x and y != y)   # noqa: E731  (NaN in both modes counts as equal)
        d["bit_identical"] = all(same(a["price"], b["price"]) and bool((a["delta"] == b["delta"]).all())
                                 for a, b in zip(res["batched"], res["plain"]))
        d["non_finite"] = sum(1 for a in res["batched"] if not math.isfinite(a["price"]))
        d["checks"] = book_checks(eng, opts, res["batched"], orv) if world == 1 else None
        d["converged"] = sum(1 for x in res["batched"] if x["converged"])
        return d

    def at_eps(opts, eps):
        out = []
        for o in opts:
            c = type(o).from_buffer_copy(o)   # copies; the arrays stay with `book`
            c.eps = eps
            out.append(c)
        return out

    def batched_only(opts, total):
        r, st = eng.book_price(opts, eng.BOOK_BATCHED) if opts else ([], {"time_s": 0.0, "rounds": 0, "launches": 0,
                                                                         "normals": 0.0, "path_steps": 0.0})
        agg = torch.tensor([st["time_s"], st["normals"], st["path_steps"]], dtype=torch.float64, device="cuda")
        if world > 1:
            t = agg[:1].clone()
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            w = agg[1:].clone()
            torch.distributed.all_reduce(w, op=torch.distributed.ReduceOp.SUM)
            agg = torch.cat([t, w])
        tmax, normals, psteps = agg.tolist()
        d = {"options": total, "batched": {"options_per_s": total / tmax, "time_s": tmax, "rounds": st["rounds"],
                                           "launches": st["launches"], "normals_per_s": normals / tmax,
                                           "path_steps_per_s": psteps / tmax}}
        d["non_finite"] = sum(1 for a in r if not math.isfinite(a["price"]))
        d["checks"] = book_checks(eng, opts, r, orv) if world == 1 else None
        d["converged"] = sum(1 for x in r if x["converged"])
        return d

    mine = [book[i] for i in range(rank, n, world)]
    out = {"options": n, "workload": "first %d of the 4096-option synthetic basket book (seed 5), %.1f %% of it; "
                                     "MLQMC R=16 M=2 n0=1, price + per-asset delta" % (n, 100.0 * n / 4096),
           "sharding": "options round-robin over %d rank(s), fixed total" % world}
    if n_all > 0:
        # the metric's configuration at (up to) its full size: every option at eps = 1e-3, batched form only
        # (the plain form of all 4096 would double the section's minutes; its ratio is measured on the prefix)
        all_mine = [book[i] for i in range(rank, n_all, world)]
        out["eps_1e-3_all"] = batched_only(at_eps(all_mine, 1e-3), n_all)
        out["eps_1e-3_all"]["workload"] = ("first %d of the 4096-option book (%.1f %% of it) at eps = 1e-3, batched"
                                           % (n_all, 100.0 * n_all / 4096))
    out["eps_1e-3"] = both_modes(at_eps(mine, 1e-3), n)
    out["own_eps"] = both_modes(mine, n)
    loose = [book[i] for i in range(rank, n_loose, world)]
    out["eps_5e-3"] = both_modes(at_eps(loose, 5e-3), n_loose)
    out["eps_5e-3"]["options"] = n_loose
    # a mixed book: the first 128 baskets with 128 single-asset options (GBM, Heston and Dupire;
    # European, Asian, lookback and down-and-out calls; 64 finest steps), each at its own eps
    singles = eng.mixed_singles(n=128, seed=6)
    mixed = [book[i] for i in range(128)] + singles
    mine_mixed = [mixed[i] for i in range(rank, len(mixed), world)]
    out["mixed"] = both_modes(mine_mixed, len(mixed))
    out["mixed"]["workload"] = ("first 128 basket options of the synthetic book with 128 single-asset options "
                                "(mixed_singles seed 6), each at its own eps")
    return out


def book_slice(spec):
    """One (option, level) slice through the book kernel: a D-asset correlated basket call
    (seeded as the synthetic book), all 16 replicas, POINTS points (default: about 4e9 normals)."""
    import numpy as np
    import torch
    parts = [int(v) for v in spec.split(":")]
    d, level = parts[0], parts[1]
    nf = 2 ** level
    n = parts[2] if len(parts) > 2 else min(max(1 << 12, int(4e9 / (16 * nf * d))), 1 << 30)
    eng = load_engine()
    eng.init(0)
    rng = np.random.default_rng(3)
    S0, sig = 100 * rng.uniform(0.8, 1.2, d), rng.uniform(0.1, 0.5, d)
    A = rng.normal(size=(d, d))
    Cm = A @ A.T + 0.5 * np.eye(d)
    dg = np.sqrt(np.diag(Cm))
    w = rng.dirichlet(np.ones(d))
    o = eng.book_option(S0, sig, float(w @ S0), 0.03, 1.0, 1e-3, max(level, 2), weights=w,
                        L=np.linalg.cholesky(Cm / np.outer(dg, dg)))
    ml, qc = eng.mlmc_cfg(M=2, n0_steps=1), eng.qmc_cfg(R=16)
    eng.book_level_sums(o, level, 0, min(n, 4096), ml, qc)
    best = float("inf")
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.book_level_sums(o, level, 0, n, ml, qc)
        best = min(best, time.perf_counter() - t0)
    normals = 16.0 * n * nf * d
    print(json.dumps({"book_slice": {"assets": d, "level": level, "points": n, "replicas": 16,
                                     "normals": normals, "seconds": best, "normals_per_s": normals / best}}))


def pass_case(name, repeats=6):
    """One fused pass of another benchmark configuration, `repeats` calls through the public API
    (the profiling cases of those kernels): `heston_level` is the config-3 coupled level pair
    (Heston kappa 2, theta 0.04, xi 0.3, rho -0.7, v0 0.04, r 0.02, Euler-Milstein variance, lookback
    call, level 4 of M = 4 and n0 = 4: 1024 fine / 256 coarse steps, 16 replicas x 2^17 scrambled
    points; the first three calls are the autotuner's trials); `philox_eur` is the config-1 plain MC pass (GBM European, S0 = K = 100, r 0.05,
    sigma 0.2, 64 steps, 2^22 Philox paths)."""
    eng = load_engine()
    eng.init(0)
    if name == "heston_level":
        m = eng.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)
        run = lambda: eng.level_pass(m, eng.lookback(0.3), 4 * 4 ** 4, 4, use_sobol=True, salt_base=42,  # noqa: E731
                                     R=16, n_points=1 << 17, flags=eng.FLAG_HESTON_MILSTEIN)
        units = 16 * (1 << 17) * (1024 + 256)
    elif name == "philox_eur":
        m = eng.gbm(100.0, 0.05, 0.2, 1.0)
        run = lambda: eng.mc_pass(m, eng.european(100.0, 0.05, 1.0), 64, 123, 0, 0, 1 << 22)  # noqa: E731
        units = (1 << 22) * 64
    else:
        raise SystemExit("unknown --pass-case " + name)
    best = float("inf")
    for _ in range(repeats):
        t0 = time.perf_counter()
        out = run()
        best = min(best, time.perf_counter() - t0)
    print(json.dumps({"pass_case": {"name": name, "seconds": best, "path_steps_per_s": units / best,
                                    "sums": [float(v) for v in out.reshape(-1)[:4]]}}))


def adjoint_case(n_points, repeats=3):
    """The config-4 adjoint (64 x 32 local-vol grid, Asian call, T 2, 512 steps, 16 replicas x
    n_points scrambled paths, price + delta + rho + 2048 node vegas), `repeats` calls through the
    public API: the profiling case of k_adjoint."""
    import torch
    eng = load_engine()
    eng.init(0)
    K, tt, grid = eng.config4_surface()
    lv = eng.localvol_grid(K, tt, grid, 100.0, 0.05, 2.0)
    best = float("inf")
    for _ in range(repeats):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g, _ = eng.adjoint(lv, eng.asian(100.0), 512, salt_base=42, R=16, n_points=n_points)
        best = min(best, time.perf_counter() - t0)
    print(json.dumps({"adjoint_case": {"paths": 16 * n_points, "seconds": best, "price": g["price"],
                                       "delta": g["delta"], "rho": g["rho"], "vega": g["vega"]}}))


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    steps = []
    cb = None
    per = max(2.0, 60.0 / max(args.steps + args.warmup, 1))
    for i in range(args.warmup + args.steps):
        c = cpu_baseline(seconds=per, steps=1)
        if i >= args.warmup:
            steps.append(c["value"])
            cb = c
    v = sorted(steps)[len(steps) // 2]
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "RQMC arithmetic Asian call, GBM S0=K=100 r=0.03 sigma=0.25 T=1, "
                                   "256 steps / Sobol dims, R=32 HH-scrambled replicas, raw ordering"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--points", type=int, default=1 << 20, help="points per replica per step")
    ap.add_argument("--e2e-runs", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true", help="skip the bridge / PCA orderings")
    ap.add_argument("--book-options", type=int, default=256,
                    help="options of the synthetic basket book priced batched and plain (0: skip)")
    ap.add_argument("--book-options-loose", type=int, default=4096,
                    help="options priced at the loosest eps of the range (5e-3)")
    ap.add_argument("--book-options-all", type=int, default=4096,
                    help="options priced batched only at the metric's eps = 1e-3 (0: skip)")
    ap.add_argument("--no-configs", action="store_true", help="skip the MC / Heston MLQMC / adjoint workloads")
    ap.add_argument("--book-slice", default=None, metavar="D:LEVEL[:POINTS]",
                    help="only price one slice of a D-asset basket at LEVEL through the book kernel "
                         "(R = 16, M = 2, n0 = 1) and print its normals/s: the profiling case")
    ap.add_argument("--pass-case", default=None, choices=["heston_level", "philox_eur"],
                    help="only run one fused pass of another configuration (the profiling cases)")
    ap.add_argument("--adjoint-case", type=int, default=None, metavar="POINTS",
                    help="only run the config-4 local-vol adjoint with 16 x POINTS paths, three times (the "
                         "profiling case of k_adjoint)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.adjoint_case:
        return adjoint_case(args.adjoint_case)
    if args.pass_case:
        return pass_case(args.pass_case)
    if args.impl == "reference":
        return run_reference(args)
    if args.book_slice:
        return book_slice(args.book_slice)

    import torch
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    eng = load_engine()
    eng.init(local_rank)
    m, p = eng.gbm(S0, R_, SIG, T_), eng.asian(K)
    salt = SALT + REPS * rank
    N = args.points
    sums = torch.zeros(REPS * 2, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # a dedicated stream: torch's default stream has handle 0, which the C ABI reads as "use
    # the engine's internal stream", and the events below must sit on the launching stream
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    assert sp != 0

    import importlib
    sharded = importlib.import_module("fdmc_b200.sharded")
    gsums = [sums]   # the estimator's [32 N][2] per-replica sums after the last pass

    def one_pass():
        eng.qmc_pass_device(m, p, STEPS, sums.data_ptr(), sp, salt_base=salt, R=REPS, offset=0, n_points=N)
        if world > 1:   # the estimator over all ranks' replicas, on every rank (NCCL on `stream`)
            gsums[0] = sharded.combine_replica_sums(sums.view(REPS, 2), world * REPS)

    # the clock sampler starts before the warm-up (nvidia-smi needs a moment to start) and its
    # summary keeps the samples from the start of the timed region on
    clk = ClockSampler(local_rank).__enter__()
    for _ in range(args.warmup):
        flush.zero_()
        one_pass()
    torch.cuda.synchronize()
    clk.wait_rows(1, 10.0)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk_first = len(clk.rows)
    for i in range(args.steps):
        flush.zero_()
        evs[i][0].record(stream)
        one_pass()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    clk.wait_rows(clk_first + 1, 2.0)   # at least the sample that closes the timed region
    clocks = clk.summary(clk_first)
    clk.__exit__(None, None, None)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = sum(ms)
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    ps_per_step = REPS * N * STEPS
    value = world * ps_per_step * args.steps / (total_ms * 1e-3)
    chk = gsums[0].cpu().numpy().reshape(world * REPS, 2)
    rmeans = chk[:, 0] / N
    price = float(rmeans.mean())
    price_se = float(rmeans.std(ddof=1) / math.sqrt(world * REPS))

    # the same workload under Brownian-bridge and PCA (tcgen05) ordering, same timing rules
    variants = {}
    if not args.no_variants:
        for name, noise in (("bridge", eng.BB), ("pca_tcgen05", eng.PCA)):
            h = eng.bb_create(STEPS, T_) if noise == eng.BB else eng.pca_create(STEPS, T_)
            kw = {"bb": h} if noise == eng.BB else {"pca": h}
            for _ in range(args.warmup):
                eng.qmc_pass_device(m, p, STEPS, sums.data_ptr(), sp, noise=noise, salt_base=salt, R=REPS,
                                    n_points=N, **kw)
            tv = 0.0
            for i in range(max(3, args.steps // 2)):
                flush.zero_()
                a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a_.record(stream)
                eng.qmc_pass_device(m, p, STEPS, sums.data_ptr(), sp, noise=noise, salt_base=salt, R=REPS,
                                    n_points=N, **kw)
                b_.record(stream)
                b_.synchronize()
                tv += a_.elapsed_time(b_)
            nv = max(3, args.steps // 2)
            vm = sums.cpu().numpy().reshape(REPS, 2)[:, 0] / N
            variants[name] = {"value": ps_per_step * nv / (tv * 1e-3), "ms_per_step": tv / nv,
                              "price": float(vm.mean()), "std_error": float(vm.std(ddof=1) / math.sqrt(REPS))}
            h.close()

    # the same workload with the geometric-average payoff, against its discrete closed form
    eng.qmc_pass_device(m, eng.geom_asian(K), STEPS, sums.data_ptr(), sp, salt_base=salt, R=REPS, offset=0,
                        n_points=N)
    torch.cuda.synchronize()
    gm = sums.cpu().numpy().reshape(REPS, 2)[:, 0] / N
    geom_check = {"price": float(gm.mean()), "std_error": float(gm.std(ddof=1) / math.sqrt(REPS))}

    # e2e: the reference-facing adaptive driver with host structs (one rank), or the same doubling
    # loop with the replicas split over the ranks (host buffers through mcq_qmc_pass per block)
    cfg = eng.qmc_cfg(R=REPS, N0_per_replica=1 << 14, salt_base=salt)
    if world == 1:
        def e2e_run():
            r = eng.run_qmc(m, p, 1e-3, STEPS, cfg)
            return r, r["path_steps"]
    else:
        def e2e_run():
            def pass_fn(r0, nr, offset, n):
                return eng.qmc_pass(m, p, STEPS, salt_base=SALT + r0, R=nr, offset=offset, n_points=n)
            r = sharded.run_qmc_sharded(pass_fn, world * REPS, 1e-3, 1 << 14, max_doublings=cfg.max_doublings,
                                        device="cuda")
            lo, hi = sharded.replica_block(world * REPS, world, rank)
            return r, float(r["n_samples"]) / (world * REPS) * (hi - lo) * STEPS
    e2e_run()   # warm-up (tables, streams)
    e2e_ps, e2e_t, e2e_last = 0.0, 0.0, None
    for _ in range(args.e2e_runs):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r, ps = e2e_run()
        e2e_t += time.perf_counter() - t0
        e2e_ps += ps
        e2e_last = r
    if world > 1:
        t = torch.tensor([e2e_t, e2e_ps], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t[:1], op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(t[1:], op=torch.distributed.ReduceOp.SUM)
        e2e_t, e2e_ps = float(t[0].item()), float(t[1].item())
    e2e_value = e2e_ps / e2e_t
    doublings = max(1, int(round(math.log2(e2e_last["n_samples"] / (world * REPS << 14)))) + 1)
    import ctypes
    h2d_e2e = ctypes.sizeof(m) + ctypes.sizeof(p) + ctypes.sizeof(cfg)

    orv = oracle_values()
    book = None if args.book_options <= 0 else book_bench(eng, args.book_options, args.book_options_loose, orv,
                                                          args.book_options_all)
    others = None if args.no_configs else configs_bench(eng, orv)

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    peaks = measured_peaks()
    sm_count = torch.cuda.get_device_properties(local_rank).multi_processor_count
    mhz = clocks["sm_mhz"] or peaks.get("clocks_under_load", {}).get("sm_mhz_median") or 1965.0
    peak_fp32 = sm_count * 128 * 2 * mhz * 1e6 / 1e12
    per_launch_ms = total_ms / args.steps
    achieved = ps_per_step * FLOPS_PER_PATH_STEP / (per_launch_ms * 1e-3) / 1e12
    traffic, issue = None, None
    try:   # DRAM bytes of one launch and issue activity from the committed ncu capture
        with open(os.path.join(ROOT, "profiles", "traffic_k_pass.json")) as f:
            tj = json.load(f)
        traffic, issue = tj["dram_bytes_per_launch"], tj.get("issue_active")
    except (OSError, ValueError, KeyError):
        pass
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "RQMC arithmetic Asian call, GBM S0=K=100 r=0.03 sigma=0.25 T=1, 256 steps "
                               "= 256 Sobol dims, R=32 HH-scrambled replicas, raw ordering",
                   "points_per_replica_per_step": N, "replicas_per_gpu": REPS, "global_batch": world * REPS * N,
                   "seq_len": STEPS, "parallelism": f"replicas x{world}" if world > 1 else "single",
                   "l2": "flushed (256 MiB write) between steps; inputs are parameter-sized"},
        "price_check": price,
        "price_check_se": price_se,
        "vs_oracle": vs_oracle(price, price_se, orv.get("asian_gbm_256", {}).get("value"),
                               orv.get("asian_gbm_256", {}).get("se", 0.0), orv.get("asian_gbm_256", {}).get("kind", "")),
        "geom_check": dict(geom_check, vs_closed_form=vs_oracle(
            geom_check["price"], geom_check["std_error"], orv.get("asian_gbm_256", {}).get("geom_closed_form"), 0.0,
            "discrete geometric-Asian closed form (256 monitoring dates); includes the Euler scheme's bias")),
        "orderings": {k: dict(v, vs_oracle=vs_oracle(v["price"], v["std_error"],
                                                     orv.get("asian_gbm_256", {}).get("value"),
                                                     orv.get("asian_gbm_256", {}).get("se", 0.0),
                                                     orv.get("asian_gbm_256", {}).get("kind", "")))
                      for k, v in variants.items()},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d_e2e,
                "d2h_bytes_per_step": doublings * REPS * 2 * 8,
                "what": "mcq_run_qmc (run_qmc_cuda entry) eps=1e-3 from 2^14 pts/replica, host wall time; a step "
                        "is one driver call: its inputs are the host model / payoff / config structs (copied to "
                        "the device as kernel parameters, counted in h2d), its outputs the per-replica sums of "
                        "each doubling read back (d2h)",
                "price": e2e_last["price"], "std_error": e2e_last["std_error"], "n_samples": e2e_last["n_samples"],
                "converged": bool(e2e_last["converged"]),
                "vs_oracle": vs_oracle(e2e_last["price"], e2e_last["std_error"],
                                       orv.get("asian_gbm_256", {}).get("value"), orv.get("asian_gbm_256", {}).get("se", 0.0),
                                       orv.get("asian_gbm_256", {}).get("kind", "")),
                "path_steps_per_run": e2e_last["path_steps"], "ms_per_run": 1e3 * e2e_t / args.e2e_runs},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak_fp32, "unit": "TFLOP/s",
                     "frac": achieved / peak_fp32, "traffic": traffic,
                     "peak_source": f"derived: {sm_count} SMs x 128 FP32 lanes x 2 x {mhz:.0f} MHz (median SM clock "
                                    "sampled under load); MEASURED_PEAKS.json has no FP32 figure",
                     "flops_per_path_step": FLOPS_PER_PATH_STEP, "sfu_per_path_step": SFU_PER_PATH_STEP,
                     "kernel": "k_pass<Sobol, raw, PathC<GBM, Asian>>",
                     "issue_model": {"flops_per_path_step": ISSUE_MODEL_FLOPS_PER_PATH_STEP,
                                     "achieved": achieved * ISSUE_MODEL_FLOPS_PER_PATH_STEP / FLOPS_PER_PATH_STEP,
                                     "frac": achieved * ISSUE_MODEL_FLOPS_PER_PATH_STEP / FLOPS_PER_PATH_STEP / peak_fp32,
                                     "what": "the inverse normal counted as the 29-flop AS241 rational"},
                     "issue_active_ncu": issue,
                     "instructions_per_path_step_ncu": 37.7,
                     "note": "instruction-issue bound: the algorithmic count is 13 FP32 flops and one inverse "
                             "normal per path-step, the kernel issues about 38 thread instructions per path-step "
                             "(about 24 in CUDA's normcdfinvf, 3 in the GBM step and Asian sum, 10 in the Sobol "
                             "generation and transpose) at the issue activity of the committed ncu capture"},
        "gpu_launches": 2 * args.steps,
        "clocks": clocks,
    }
    if book is not None:
        line["book"] = book
    if others is not None:
        line["other_workloads"] = others
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
