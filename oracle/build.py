"""Build recipe for the oracle (test infrastructure only).

Compiles oracle/oracle.c (CPU restatement of the LAPACK algorithms the
reference tests against), oracle/refgen.cpp (the reference client's integer
generator) and oracle/lapack_host.c (host LAPACK over a batch, loaded with dlopen:
the timed CPU baseline) into oracle/_build/liboracle.so.  The product library never links
this; only tests/, __graft_entry__.smoke() and bench.py's CPU baseline load it.

The reference itself (HIP + rocBLAS, AMD GPUs only) cannot be compiled here, so
there is no oracle/_ref build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, "oracle.c"), os.path.join(HERE, "refgen.cpp"),
            os.path.join(HERE, "lapack_host.c"), os.path.join(HERE, "oracle_complex.c")]
    if not force and os.path.exists(LIB):
        lib_t = os.path.getmtime(LIB)
        if all(os.path.getmtime(s) <= lib_t for s in srcs + [__file__]):
            return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    obj_c = os.path.join(OUT_DIR, "oracle.o")
    obj_cpp = os.path.join(OUT_DIR, "refgen.o")
    obj_lh = os.path.join(OUT_DIR, "lapack_host.o")
    obj_cx = os.path.join(OUT_DIR, "oracle_complex.o")
    # -ffp-contract=off: the restatement must round like the unfused reference BLAS loops
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-ffp-contract=off", "-std=c11", "-Wall",
                           "-c", srcs[0], "-o", obj_c])
    subprocess.check_call(["g++", "-O2", "-fPIC", "-std=c++17", "-Wall", "-c", srcs[1],
                           "-o", obj_cpp])
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-std=c11", "-Wall", "-c", srcs[2],
                           "-o", obj_lh])
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-ffp-contract=off", "-std=c11", "-Wall",
                           "-c", srcs[3], "-o", obj_cx])
    tmp = LIB + ".tmp"
    subprocess.check_call(["g++", "-shared", "-o", tmp, obj_c, obj_cpp, obj_lh, obj_cx, "-lm",
                           "-lpthread", "-ldl"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
