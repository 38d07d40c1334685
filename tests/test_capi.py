"""C-ABI boundary checks that need no GPU: the library loads, exports every symbol
include/mcq.h declares, links nothing from the oracle, and rejects bad arguments with status
codes (never exceptions or crashes) before it touches the device."""
import ctypes as C
import os
import re
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "mcq.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mcq_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported(eng):
    L = eng.lib()
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(eng.EXPORTS)


def test_library_does_not_link_the_oracle(eng):
    out = subprocess.run(["readelf", "-d", eng.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in out
    syms = subprocess.run(["nm", "-D", eng.LIB_PATH], capture_output=True, text=True).stdout
    assert " orc_" not in syms


def test_version_and_defaults(eng):
    assert eng.version() == 100
    mc, qc, ml = eng.mc_cfg(), eng.qmc_cfg(), eng.mlmc_cfg()
    # methods_cuda.cuh:10-32 defaults
    assert (mc.N_batch, mc.pilot_n, mc.seed) == (1 << 16, 10000, 123)
    assert (qc.R, qc.max_doublings, qc.salt_base, qc.N0_per_replica) == (32, 20, 42, 0)
    assert (ml.M, ml.max_L, ml.pilot_n, ml.n0_steps) == (2, 10, 400, 1)


def test_heston_helper_fills_cholesky(eng):
    m = eng.mcq_types.Model()
    assert eng.lib().mcq_model_heston(C.c_double(100), C.c_double(0.02), C.c_double(2), C.c_double(0.04),
                                      C.c_double(0.3), C.c_double(-0.7), C.c_double(0.04), C.c_double(1),
                                      C.byref(m)) == 0
    assert m.kind == eng.HESTON and m.hes_L10 == -0.7 and abs(m.hes_L11 - np.sqrt(1 - 0.49)) < 1e-15


def test_host_philox_matches_oracle(eng, orc):
    for ctr, key in (([0, 0, 0, 0], [0, 0]), ([1, 2, 3, 4], [123, 0x6D637121]), ([0xffffffff] * 4, [7, 9])):
        assert eng.philox(ctr, key) == orc.philox(ctr, key)


def test_null_and_bad_arguments_return_status(eng):
    L = eng.lib()
    r = eng.mcq_types.Result()
    m, p = eng.gbm(), eng.european(100, 0.05, 1)
    assert L.mcq_run_qmc(None, C.byref(p), C.c_double(1e-3), 64, None, 0, None, None, C.byref(r)) == 1
    assert b"NULL" in L.mcq_last_error()
    assert L.mcq_run_mc(C.byref(m), None, C.c_double(1e-3), 64, None, C.byref(r)) == 1
    h = C.c_void_p()
    assert L.mcq_bb_create(3, C.c_double(1.0), C.byref(h)) == 1          # N not a power of two
    assert L.mcq_bb_create(8, C.c_double(-1.0), C.byref(h)) == 1         # T <= 0
    assert L.mcq_pca_create(0, C.c_double(1.0), C.byref(h)) == 1
    assert L.mcq_sobol_hh_u32(42, 0, 1, 0, 10, None) == 1
    out = np.zeros(10, np.uint32)
    p32 = out.ctypes.data_as(C.POINTER(C.c_uint32))
    assert L.mcq_sobol_hh_u32(42, 19999, 2, 0, 10, p32) == 4             # dims beyond the table
    assert L.mcq_sobol_hh_u32(42, 0, 1, C.c_uint32(0xFFFFFFF0), C.c_int64(100), p32) == 4  # index beyond 2^32
    assert L.mcq_philox4x32_10(None, None, None) == 1
    assert L.mcq_debug_wait_timeout(C.c_uint32(0)) == 1                   # polls out of range
    assert L.mcq_debug_wait_timeout(C.c_uint32(1 << 21)) == 1


def test_error_message_is_thread_local(eng):
    import threading
    L = eng.lib()
    msgs = {}

    def worker(i):
        L.mcq_bb_create(3 + 2 * i, C.c_double(1.0), C.byref(C.c_void_p()))
        msgs[i] = L.mcq_last_error()

    ts = [threading.Thread(target=worker, args=(i,)) for i in range(4)]
    [t.start() for t in ts]
    [t.join() for t in ts]
    assert all(b"power of two" in v for v in msgs.values())
