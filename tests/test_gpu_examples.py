"""The reference's own example programs (examples/ejemplo01..11) run end to end on the engine: each
is compiled from its unchanged source against include/mcq.hpp (the reference's C++ API over the C
ABI) by `make -C oracle examples` where the reference is present, and the built programs run
here.  Each program estimates c1 by Richardson (estimar_c1_richardson), sizes its step count from
it, runs its MC / MLMC / QMC / MLQMC / CV / IS drivers and prints the reference's table; the
table is read back with the reference report script's regexes (gen_informe.py:16-21).  The
reference's own check of a row is |price - reference| < 2 eps (SI); a driver's result carries its
statistical error besides the bias its step count was sized for, so every row must be within
2 eps + 2 SE of the reference: SI, or NO by less than two standard errors (e.g. ejemplo02's pseudo-random MC row at the default eps: bias ~0.07 plus one SE of 0.035
against 2 eps = 0.1).  Programs that are not built are skipped."""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EX = os.path.join(ROOT, "oracle", "_ref", "examples")
NAMES = ["ejemplo01_european", "ejemplo02_asian", "ejemplo03_lookback", "ejemplo04_barrier", "ejemplo05_heston",
         "ejemplo06_dupire", "ejemplo07_basket_uncorr", "ejemplo08_basket_corr", "ejemplo09_asian_cv",
         "ejemplo10_dupire_cv", "ejemplo11_otm_is"]

# gen_informe.py:20-21
REF_RE = re.compile(r"Referencia:\s*([\d.]+)")
ROW_RE = re.compile(r"^\s{2}(.+?)\s+([\d.]+)\s+([\d.]+)\s+(\d+)\s+([\d.]+)\s+([\d.]+)\s+(SI|NO)\s*$")


@pytest.mark.parametrize("name", NAMES)
def test_reference_example_runs_on_engine(name):
    exe = os.path.join(EX, name)
    if not os.path.exists(exe):
        pytest.skip("reference examples not built (make -C oracle examples needs the reference sources)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    out = r.stdout
    m = REF_RE.search(out)
    assert m, out
    rows = [ROW_RE.match(ln) for ln in out.splitlines()]
    rows = [x for x in rows if x]
    assert len(rows) >= 2, out
    eps = float(re.search(r"epsilon = ([\d.eE+-]+)", out).group(1))
    for x in rows:
        assert int(x.group(4)) > 0 and float(x.group(3)) >= 0.0
        err, se = float(x.group(6)), float(x.group(3))
        assert err < 2 * eps + 2 * se, (x.group(0), out)   # SI, or NO by less than 2 SE
