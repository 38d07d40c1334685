"""Build libmcq.so (the engine) for sm_100a with nvcc, in-tree.

Compiles every translation unit under csrc/ in parallel into ../_build/ and links
financial-derivatives-montecarlo_b200/libmcq.so.  Usage: python build.py [--force] [-j N].
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(ROOT, "_build", "mcq")
LIB = os.path.join(HERE, "libmcq.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = shutil.which("nvcc") or os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", os.path.join(ROOT, "include")]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "mcq.h"))
    return max(os.path.getmtime(h) for h in hs)


def compile_one(src, force, verbose_ptxas):
    obj = os.path.join(BUILD, src + ".o")
    s = os.path.join(CSRC, src)
    if not force and os.path.exists(obj) and os.path.getmtime(obj) > max(os.path.getmtime(s), headers_mtime()):
        return src, True, ""
    cmd = [NVCC] + ARCH + COMMON + ["-c", s, "-o", obj]
    if src.endswith(".cu") and verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode == 0, r.stdout + r.stderr


def build(force=False, jobs=None, verbose_ptxas=False, quiet=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    jobs = jobs or max(1, os.cpu_count() or 1)
    logs = {}
    with cf.ThreadPoolExecutor(jobs) as ex:
        for src, ok, log in ex.map(lambda s: compile_one(s, force, verbose_ptxas), srcs):
            logs[src] = log
            if not ok:
                sys.stderr.write(log)
                raise RuntimeError("nvcc failed on " + src)
    objs = [os.path.join(BUILD, s + ".o") for s in srcs]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-L", os.path.join(CUDA, "lib64"), "-lcurand", "-lcublas", "-Xlinker", "-rpath," + os.path.join(CUDA, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    if not quiet:
        print("built", LIB)
    return logs


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--ptxas", action="store_true", help="print register / spill report")
    a = ap.parse_args()
    logs = build(a.force, a.j, a.ptxas)
    if a.ptxas:
        for k, v in logs.items():
            print("==", k)
            print(v)
