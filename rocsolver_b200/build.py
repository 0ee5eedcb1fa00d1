"""Build librocsolver_b200.so in-tree with nvcc for sm_100a.

    python -m rocsolver_b200.build [--force] [--verbose] [--checked]

Sources: rocsolver_b200/csrc/*.cu and *.cpp.  Objects go to rocsolver_b200/_build/, the
shared library to rocsolver_b200/librocsolver_b200.so (loaded by rocsolver_b200/__init__.py).
--checked builds the bounds-checked variant instead (-DRSB_BOUNDS_CHECK: every element
access of the factor and solve kernels checked, violations recorded for
rocsolver_b200_bounds_check) into rocsolver_b200/_build_checked/ and
rocsolver_b200/librocsolver_b200_checked.so.
"""
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librocsolver_b200.so")
CHECKED_LIB = os.path.join(HERE, "librocsolver_b200_checked.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
                  + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, checked=False):
    bdir = BUILD + "_checked" if checked else BUILD
    lib = CHECKED_LIB if checked else LIB
    flags = NVCC_FLAGS + (["-DRSB_BOUNDS_CHECK"] if checked else [])
    os.makedirs(bdir, exist_ok=True)
    srcs = _sources()
    hdrs = _headers() + [os.path.abspath(__file__)]
    objs = []
    jobs = []
    for s in srcs:
        o = os.path.join(bdir, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [_nvcc()] + ARCH + flags + ["-c", s, "-o", o]
            if verbose and s.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    failed = False
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode != 0 or verbose:
                sys.stderr.write(" ".join(cmd[-3:]) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                failed = True
    if failed:
        raise RuntimeError("nvcc failed")
    if force or jobs or _stale(lib, objs):
        tmp = lib + ".tmp"
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart_static", "-lrt",
                                                                   "-lpthread", "-ldl"]
        subprocess.check_call(cmd)
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv,
                checked="--checked" in sys.argv))
