"""ctypes front end of the oracle (TEST INFRASTRUCTURE ONLY).

Wraps oracle/oracle.c for numpy arrays.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg import this module; the product library never
does.  All matrices are column-major numpy arrays of shape (batch, ld, ncols)
stored as ``a[b].T`` views are avoided: we keep an explicit Fortran layout by
passing flat buffers with (ld, stride) like the reference API.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None

OP_GETRF, OP_GETRS, OP_POTRF, OP_POTRS, OP_GESV, OP_POSV = range(6)


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        l = ctypes.CDLL(path)
        l.oracle_batch.restype = None
        l.oracle_batch.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
            ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
            ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        l.refgen_fill.restype = None
        l.refgen_fill.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        _lib = l
    return _lib


def _ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def _dbl(a):
    if a.dtype == np.float64:
        return 1
    if a.dtype == np.float32:
        return 0
    raise TypeError(a.dtype)


def nthreads_default():
    return max(1, os.cpu_count() or 1)


# Flat-buffer API mirroring the strided-batched reference signatures.  Arrays are
# 1-D numpy buffers; member b of A starts at b*strideA (elements).

def getrf(m, n, A, lda, strideA, ipiv, strideP, info, bc, pivot=True, nthreads=1):
    lib().oracle_batch(OP_GETRF, _dbl(A), m, n, 0, 0, 0, int(pivot), _ptr(A), lda, strideA,
                       _ptr(ipiv), strideP, None, 0, 0, _ptr(info), bc, nthreads)


def getrs(trans, n, nrhs, A, lda, strideA, ipiv, strideP, B, ldb, strideB, bc, nthreads=1):
    lib().oracle_batch(OP_GETRS, _dbl(A), n, n, nrhs, int(bool(trans)), 0, 1, _ptr(A), lda,
                       strideA, _ptr(ipiv), strideP, _ptr(B), ldb, strideB, None, bc, nthreads)


def potrf(upper, n, A, lda, strideA, info, bc, nthreads=1):
    lib().oracle_batch(OP_POTRF, _dbl(A), n, n, 0, 0, int(upper), 0, _ptr(A), lda, strideA,
                       None, 0, None, 0, 0, _ptr(info), bc, nthreads)


def potrs(upper, n, nrhs, A, lda, strideA, B, ldb, strideB, bc, nthreads=1):
    lib().oracle_batch(OP_POTRS, _dbl(A), n, n, nrhs, 0, int(upper), 0, _ptr(A), lda, strideA,
                       None, 0, _ptr(B), ldb, strideB, None, bc, nthreads)


def gesv(n, nrhs, A, lda, strideA, ipiv, strideP, B, ldb, strideB, info, bc, nthreads=1):
    lib().oracle_batch(OP_GESV, _dbl(A), n, n, nrhs, 0, 0, 1, _ptr(A), lda, strideA, _ptr(ipiv),
                       strideP, _ptr(B), ldb, strideB, _ptr(info), bc, nthreads)


def posv(upper, n, nrhs, A, lda, strideA, B, ldb, strideB, info, bc, nthreads=1):
    lib().oracle_batch(OP_POSV, _dbl(A), n, n, nrhs, 0, int(upper), 0, _ptr(A), lda, strideA,
                       None, 0, _ptr(B), ldb, strideB, _ptr(info), bc, nthreads)


def refgen(count):
    """Reference client's integer stream (mt19937(69069), uniform_int 1..10)."""
    out = np.empty(count, dtype=np.float64)
    lib().refgen_fill(_ptr(out), count)
    return out
