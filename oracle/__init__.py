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

OP_GETRF, OP_GETRS, OP_POTRF, OP_POTRS, OP_GESV, OP_POSV, OP_GETRI = range(7)


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


def getri(n, A, lda, strideA, ipiv, strideP, info, bc, pivot=True, nthreads=1):
    """Inverse from the LU factors (LAPACK dgetri); A overwritten where info == 0."""
    lib().oracle_batch(OP_GETRI, _dbl(A), n, n, 0, 0, 0, int(pivot), _ptr(A), lda, strideA,
                       _ptr(ipiv), strideP, None, 0, 0, _ptr(info), bc, nthreads)


# ---- complex (c/z): complex64 / complex128 numpy buffers; op 0 getrf, 1 getrs (trans 0 N,
# 1 T, 2 C), 2 potrf, 3 potrs, 4 gesv, 5 posv, 6 getri (oracle/oracle_complex.c)
def _cbatch(op, A, m=0, n=0, nrhs=0, trans=0, upper=0, pivot=1, lda=1, sA=0, ipiv=None, sP=0,
            B=None, ldb=1, sB=0, info=None, bc=1):
    l = lib()
    if A.dtype == np.complex128:
        f = l.oracle_zbatch
    elif A.dtype == np.complex64:
        f = l.oracle_cbatch
    else:
        raise TypeError(A.dtype)
    f.restype = None
    f.argtypes = [ctypes.c_int] * 7 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
                                       ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                       ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int]
    f(op, m, n, nrhs, trans, upper, pivot, _ptr(A), lda, sA, _ptr(ipiv), sP, _ptr(B), ldb, sB,
      _ptr(info), bc)


def cgetrf(m, n, A, lda, strideA, ipiv, strideP, info, bc, pivot=True):
    _cbatch(0, A, m, n, 0, 0, 0, int(pivot), lda, strideA, ipiv, strideP, None, 1, 0, info, bc)


def cgetrs(trans, n, nrhs, A, lda, strideA, ipiv, strideP, B, ldb, strideB, bc):
    _cbatch(1, A, n, n, nrhs, trans, 0, 1, lda, strideA, ipiv, strideP, B, ldb, strideB, None, bc)


def cpotrf(upper, n, A, lda, strideA, info, bc):
    _cbatch(2, A, n, n, 0, 0, int(upper), 0, lda, strideA, None, 0, None, 1, 0, info, bc)


def cpotrs(upper, n, nrhs, A, lda, strideA, B, ldb, strideB, bc):
    _cbatch(3, A, n, n, nrhs, 0, int(upper), 0, lda, strideA, None, 0, B, ldb, strideB, None, bc)


def cgesv(n, nrhs, A, lda, strideA, ipiv, strideP, B, ldb, strideB, info, bc):
    _cbatch(4, A, n, n, nrhs, 0, 0, 1, lda, strideA, ipiv, strideP, B, ldb, strideB, info, bc)


def cposv(upper, n, nrhs, A, lda, strideA, B, ldb, strideB, info, bc):
    _cbatch(5, A, n, n, nrhs, 0, int(upper), 0, lda, strideA, None, 0, B, ldb, strideB, info, bc)


def cgetri(n, A, lda, strideA, ipiv, strideP, info, bc, pivot=True):
    """Inverse from the LU factors (LAPACK zgetri / cgetri); A overwritten where info == 0."""
    _cbatch(6, A, n, n, 0, 0, 0, int(pivot), lda, strideA, ipiv, strideP, None, 1, 0, info, bc)


def refgen(count):
    """Reference client's integer stream (mt19937(69069), uniform_int 1..10)."""
    out = np.empty(count, dtype=np.float64)
    lib().refgen_fill(_ptr(out), count)
    return out


# ---------------------------------------------------------------------------------------
# Host LAPACK (OpenBLAS as bundled with scipy, loaded with dlopen by oracle/lapack_host.c):
# the reference's own CPU path for these routines, timed as the CPU baseline.  One LAPACK
# call per member on one thread, the batch split statically over nthreads pthreads.
(LH_GETRF_GETRS, LH_POTRF_POTRS, LH_GESV, LH_DSGESV, LH_ADJOINT, LH_GETRI, LH_VGESV,
 LH_ZGESV) = range(8)
_lh_ready = False


def lapack_library_path():
    """Path of scipy's bundled OpenBLAS (libscipy_openblas*.so), or None."""
    import glob
    try:
        import scipy
    except ImportError:
        return None
    d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))
    return cands[0] if cands else None


def lapack_available():
    global _lh_ready
    if _lh_ready:
        return True
    path = lapack_library_path()
    if path is None:
        return False
    l = lib()
    l.lapack_host_open.restype = ctypes.c_int
    l.lapack_host_open.argtypes = [ctypes.c_char_p]
    l.lapack_host_batch.restype = ctypes.c_int
    l.lapack_host_batch.argtypes = [
        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
        ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
        ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    l.lapack_host_outer.restype = ctypes.c_int
    l.lapack_host_outer.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    _lh_ready = l.lapack_host_open(path.encode()) == 0
    return _lh_ready


def lapack_library_name():
    path = lapack_library_path()
    return os.path.basename(path) if path else None


def lapack_batch(op, n, nrhs, A, lda, sA, ipiv=None, sP=0, B=None, ldb=1, sB=0, X=None, ldx=1,
                 sX=0, info=None, iter=None, nv=None, rv=None, ld=1, bc=1, nthreads=1):
    """Host LAPACK over members 0..bc-1 (flat float64 buffers, member b at b*stride)."""
    if not lapack_available():
        raise RuntimeError("host LAPACK (scipy's OpenBLAS) not available")
    r = lib().lapack_host_batch(op, n, nrhs, _ptr(A), lda, sA, _ptr(ipiv), sP, _ptr(B), ldb, sB,
                                _ptr(X), ldx, sX, _ptr(info), _ptr(iter), _ptr(nv), _ptr(rv), ld,
                                bc, nthreads)
    if r != 0:
        raise RuntimeError("lapack_host_batch failed")


def lapack_outer(n, nrhs, gB, X, gA, bc, nthreads=1):
    """gA = -gB X^T per member with host dgemm (gB, X: n x nrhs, gA: n x n, ld n)."""
    if not lapack_available():
        raise RuntimeError("host LAPACK (scipy's OpenBLAS) not available")
    if lib().lapack_host_outer(n, nrhs, _ptr(gB), _ptr(X), _ptr(gA), bc, nthreads) != 0:
        raise RuntimeError("lapack_host_outer failed")


def physical_cores():
    """Physical cores of this host (distinct (physical id, core id) pairs in /proc/cpuinfo),
    else the logical CPU count."""
    try:
        pairs, phys, core = set(), None, None
        with open("/proc/cpuinfo") as f:
            for ln in f:
                k, _, v = ln.partition(":")
                k = k.strip()
                if k == "physical id":
                    phys = v.strip()
                elif k == "core id":
                    core = v.strip()
                elif not k and phys is not None and core is not None:
                    pairs.add((phys, core))
                    phys = core = None
        if phys is not None and core is not None:
            pairs.add((phys, core))
        return len(pairs) or nthreads_default()
    except OSError:
        return nthreads_default()


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None
