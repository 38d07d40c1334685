"""The reference's own example programs compile and link unchanged against include/mcq.hpp and
libmcq.so (the drop-in claim for C++ callers).  Each example is built from a scratch copy whose
`../methods_cuda.cuh` is a one-line shim including mcq.hpp; nothing of the reference is kept.
Skipped where the reference sources are absent (their location: $MCQ_REFERENCE_DIR, default
/root/reference)."""
import glob
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_EX = os.path.join(os.environ.get("MCQ_REFERENCE_DIR", "/root/reference"), "examples")
LIBDIR = os.path.join(ROOT, "financial-derivatives-montecarlo_b200")


@pytest.mark.skipif(not os.path.isdir(REF_EX), reason="reference examples not present")
@pytest.mark.parametrize("src", sorted(glob.glob(os.path.join(REF_EX, "*.cpp"))) if os.path.isdir(REF_EX) else [])
def test_example_compiles_against_engine(src):
    with tempfile.TemporaryDirectory() as d:
        os.makedirs(os.path.join(d, "examples"))
        with open(os.path.join(d, "methods_cuda.cuh"), "w") as f:
            f.write('#include "mcq.hpp"\n')
        dst = os.path.join(d, "examples", os.path.basename(src))
        shutil.copy(src, dst)
        exe = os.path.join(d, "a.out")
        cmd = ["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"), dst, "-o", exe,
               "-L", LIBDIR, "-lmcq", "-Wl,-rpath," + LIBDIR]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]
