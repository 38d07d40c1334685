"""The caller-side helpers restated in include/mcq.hpp from the reference's utils.cpp, run through
a small C++ driver (tests/cpp/host_helpers.cpp) on the CPU:

* estimar_c1_richardson (utils.cpp:174-185): c1 = 1 / (|P(n/M) - P(n)| / (h (M - 1))) with
  n = max(4 M, 4), h = T / n, the coarse run on seed + 1, clamped at 1e-12 — the value the examples
  turn into n_steps (examples/ejemplo01_european.cpp:28-30);
* print_table (utils.cpp:192-210): the byte layout of each row
  "  {:<22}{:>10.4f}{:>10.4f}{:>12}{:>9.3f}{:>10.4f}{:>6}", and that the reference's report script
  reads it back: its row, reference and example regexes (gen_informe.py:16-21) restated here."""
import math
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "financial-derivatives-montecarlo_b200")

# gen_informe.py:20-21 (the reference line and the method row of a table)
REF_RE = re.compile(r"Referencia:\s*([\d.]+)")
ROW_RE = re.compile(r"^\s{2}(.+?)\s+([\d.]+)\s+([\d.]+)\s+(\d+)\s+([\d.]+)\s+([\d.]+)\s+(SI|NO)\s*$")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("helpers") / "host_helpers")
    cmd = ["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp",
           "host_helpers.cpp"), "-o", exe, "-L", LIBDIR, "-lmcq", "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def run(exe, what):
    r = subprocess.run([exe, what], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    return r.stdout


def test_richardson_c1_follows_the_reference_formula(driver):
    a, b, c, seed = 10.0, 3.0, 1e-3, 7
    lines = run(driver, "richardson").strip().splitlines()
    for ln in lines[:-1]:
        T, M, got = ln.split()
        T, M, got = float(T), int(M), float(got)
        n_fine = max(4 * M, 4)
        n_coarse = n_fine // M
        Pf = a + b / n_fine + c * seed
        Pc = a + b / n_coarse + c * (seed + 1)
        cb = abs(Pc - Pf) / ((T / n_fine) * (M - 1))
        assert got == pytest.approx(1.0 / max(cb, 1e-12), rel=1e-15), (T, M)
        # the step count the examples derive from it (ejemplo01_european.cpp:28-30) at eps = 0.05
        eps = 0.05
        ns = max(1, math.ceil(math.sqrt(2.0) * T / (eps * got)))
        assert 1 <= ns
    assert float(lines[-1].split()[1]) == pytest.approx(1e12)


def test_print_table_layout_and_report_parse(driver):
    out = run(driver, "table")
    rows = [("MC", 10.4526, 0.00498, 4120904, 0.110), ("MLQMC Raw", 10.4504, 0.00033, 141721, 0.637),
            ("QMC PCA", 10.3, 0.012, 1048576, 12.5),
            ("Metodo nombre largo", 99.123456, 1.5, 12345678901, 1234.5678)]
    ref, eps = 10.450584, 0.05
    lines = out.splitlines()
    assert "[Ejemplo de prueba]   epsilon = 0.05" in lines
    assert "  Referencia: 10.450584" in lines
    assert "  {:<22}{:>10}{:>10}{:>12}{:>9}{:>10}{:>6}".format("Metodo", "Precio", "StdErr", "N", "T(s)", "|Error|",
                                                             "OK?") in lines
    assert "  " + "-" * 79 in lines
    m = REF_RE.search(out)
    assert m and float(m.group(1)) == ref
    parsed = [ROW_RE.match(ln) for ln in lines]
    parsed = [p for p in parsed if p]
    assert len(parsed) == len(rows)
    for (name, price, se, n, t), p in zip(rows, parsed):
        err = abs(price - ref)
        want = "  {:<22}{:>10.4f}{:>10.4f}{:>12}{:>9.3f}{:>10.4f}{:>6}".format(name, price, se, n, t, err,
                                                                             "SI" if err < 2 * eps else "NO")
        assert p.group(0) == want
        assert p.group(1).strip() == name and int(p.group(4)) == n
        assert float(p.group(2)) == round(price, 4) and p.group(7) == ("SI" if err < 2 * eps else "NO")
