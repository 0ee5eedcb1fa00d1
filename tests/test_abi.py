"""C-ABI boundary tests that need no GPU: the library loads, exports every entry point
the public header declares, the header is valid C, and argument checking follows the
reference's order (clients/include/testing_getf2_getrf.hpp:15-111, testing_getrs.hpp,
testing_potf2_potrf.hpp, testing_potrs.hpp, testing_gesv.hpp, testing_posv.hpp *_bad_arg
functions).  None of these calls reaches a kernel launch."""
import ctypes
import os
import re
import subprocess

import pytest

import rocsolver_b200 as rs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rocsolver.h")

FAKE = ctypes.c_void_p(0x1000)  # non-null "device" pointer; never dereferenced here
NULL = None


def header_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"ROCSOLVER_EXPORT\s+[\w\s\*]+?\b(\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = rs.lib()
    syms = header_symbols()
    assert len(syms) >= 42 + 13
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", rs.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    assert not [s for s in syms if s not in exported]


def test_python_mirror_declares_every_symbol():
    assert sorted(set(rs.entry_points())) == header_symbols()


def test_header_is_c_and_cxx():
    subprocess.run(["gcc", "-fsyntax-only", "-Wall", "-x", "c", HEADER], check=True)
    subprocess.run(["g++", "-fsyntax-only", "-Wall", "-x", "c++", HEADER], check=True)


def test_version_string():
    n = ctypes.c_size_t()
    assert rs.call("rocsolver_get_version_string_size", ctypes.byref(n)) == rs.SUCCESS
    buf = ctypes.create_string_buffer(n.value)
    assert rs.call("rocsolver_get_version_string", buf, n.value) == rs.SUCCESS
    assert buf.value.decode().startswith("3.23")


@pytest.fixture
def handle():
    h = rs.Handle()
    yield h.value
    h.close()


@pytest.mark.parametrize("p", ["s", "d", "c", "z"])
def test_getrf_bad_args(handle, p):
    f = f"rocsolver_{p}getrf_strided_batched"
    # m, n, A, lda, strideA, ipiv, strideP, info, bc
    ok = dict(m=1, n=1, A=FAKE, lda=1, sA=1, ipiv=FAKE, sP=1, info=FAKE, bc=1)

    def c(h=handle, **kw):
        a = dict(ok, **kw)
        return rs.call(f, h, a["m"], a["n"], a["A"], a["lda"], a["sA"], a["ipiv"], a["sP"],
                       a["info"], a["bc"])
    assert c(h=None) == rs.INVALID_HANDLE
    assert c(m=-1) == rs.INVALID_SIZE
    assert c(n=-1) == rs.INVALID_SIZE
    assert c(m=2, lda=1) == rs.INVALID_SIZE
    assert c(bc=-1) == rs.INVALID_SIZE
    # size errors come before pointer errors
    assert c(m=-1, A=NULL) == rs.INVALID_SIZE
    assert c(A=NULL) == rs.INVALID_POINTER
    assert c(ipiv=NULL) == rs.INVALID_POINTER
    assert c(info=NULL) == rs.INVALID_POINTER
    # quick return with zero batch: info may be null (testing_getf2_getrf.hpp:59-62)
    assert c(info=NULL, bc=0) == rs.SUCCESS
    # m*n != 0 still requires A and ipiv even with zero batch (roclapack_getf2.hpp:512-514)
    assert c(A=NULL, bc=0) == rs.INVALID_POINTER
    # npvt variant needs no ipiv
    assert rs.call(f"rocsolver_{p}getrf_npvt_strided_batched", handle, 1, 1, FAKE, 1, 1, NULL, 1) \
        == rs.INVALID_POINTER
    assert rs.call(f"rocsolver_{p}getrf_npvt_strided_batched", handle, 1, 1, NULL, 1, 1, FAKE, 0) \
        == rs.INVALID_POINTER  # m*n != 0 and A null
    assert rs.call(f"rocsolver_{p}getrf_batched", None, 1, 1, FAKE, 1, FAKE, 1, FAKE, 1) \
        == rs.INVALID_HANDLE


@pytest.mark.parametrize("p", ["s", "d", "c", "z"])
def test_getrs_bad_args(handle, p):
    f = f"rocsolver_{p}getrs_strided_batched"
    ok = dict(t=rs.OP_N, n=1, r=1, A=FAKE, lda=1, sA=1, ipiv=FAKE, sP=1, B=FAKE, ldb=1, sB=1,
              bc=1)

    def c(h=handle, **kw):
        a = dict(ok, **kw)
        return rs.call(f, h, a["t"], a["n"], a["r"], a["A"], a["lda"], a["sA"], a["ipiv"],
                       a["sP"], a["B"], a["ldb"], a["sB"], a["bc"])
    assert c(h=None) == rs.INVALID_HANDLE
    assert c(t=0) == rs.INVALID_VALUE
    assert c(t=0, n=-1) == rs.INVALID_VALUE  # enum check before sizes
    assert c(n=-1) == rs.INVALID_SIZE
    assert c(r=-1) == rs.INVALID_SIZE
    assert c(n=2, lda=1, ldb=2) == rs.INVALID_SIZE
    assert c(n=2, lda=2, ldb=1) == rs.INVALID_SIZE
    assert c(bc=-1) == rs.INVALID_SIZE
    assert c(A=NULL) == rs.INVALID_POINTER
    assert c(ipiv=NULL) == rs.INVALID_POINTER
    assert c(B=NULL) == rs.INVALID_POINTER
    assert c(r=0, B=NULL) == rs.SUCCESS  # quick return: nothing to solve
    assert c(bc=0) == rs.SUCCESS
    assert c(n=0, A=NULL, ipiv=NULL, B=NULL) == rs.SUCCESS


@pytest.mark.parametrize("p", ["s", "d", "c", "z"])
def test_gesv_bad_args(handle, p):
    f = f"rocsolver_{p}gesv_strided_batched"
    ok = dict(n=1, r=1, A=FAKE, lda=1, sA=1, ipiv=FAKE, sP=1, B=FAKE, ldb=1, sB=1, info=FAKE,
              bc=1)

    def c(h=handle, **kw):
        a = dict(ok, **kw)
        return rs.call(f, h, a["n"], a["r"], a["A"], a["lda"], a["sA"], a["ipiv"], a["sP"],
                       a["B"], a["ldb"], a["sB"], a["info"], a["bc"])
    assert c(h=None) == rs.INVALID_HANDLE
    assert c(n=-1) == rs.INVALID_SIZE
    assert c(r=-1) == rs.INVALID_SIZE
    assert c(n=2, lda=1, ldb=2) == rs.INVALID_SIZE
    assert c(bc=-1) == rs.INVALID_SIZE
    for k in ("A", "ipiv", "B", "info"):
        assert c(**{k: NULL}) == rs.INVALID_POINTER, k
    assert c(bc=0, info=NULL) == rs.SUCCESS


@pytest.mark.parametrize("p", ["s", "d", "c", "z"])
def test_potrf_potrs_posv_bad_args(handle, p):
    f = f"rocsolver_{p}potrf_strided_batched"
    assert rs.call(f, None, rs.FILL_LOWER, 1, FAKE, 1, 1, FAKE, 1) == rs.INVALID_HANDLE
    assert rs.call(f, handle, rs.FILL_FULL, 1, FAKE, 1, 1, FAKE, 1) == rs.INVALID_VALUE
    assert rs.call(f, handle, 0, -1, FAKE, 1, 1, FAKE, 1) == rs.INVALID_VALUE
    assert rs.call(f, handle, rs.FILL_LOWER, -1, FAKE, 1, 1, FAKE, 1) == rs.INVALID_SIZE
    assert rs.call(f, handle, rs.FILL_LOWER, 2, FAKE, 1, 1, FAKE, 1) == rs.INVALID_SIZE
    assert rs.call(f, handle, rs.FILL_LOWER, 1, FAKE, 1, 1, FAKE, -1) == rs.INVALID_SIZE
    assert rs.call(f, handle, rs.FILL_LOWER, 1, NULL, 1, 1, FAKE, 1) == rs.INVALID_POINTER
    assert rs.call(f, handle, rs.FILL_LOWER, 1, FAKE, 1, 1, NULL, 1) == rs.INVALID_POINTER
    assert rs.call(f, handle, rs.FILL_UPPER, 1, NULL, 1, 1, NULL, 0) == rs.INVALID_POINTER
    assert rs.call(f, handle, rs.FILL_UPPER, 1, FAKE, 1, 1, NULL, 0) == rs.SUCCESS
    g = f"rocsolver_{p}potrs_strided_batched"
    assert rs.call(g, handle, rs.FILL_FULL, 1, 1, FAKE, 1, 1, FAKE, 1, 1, 1) == rs.INVALID_VALUE
    assert rs.call(g, handle, rs.FILL_LOWER, 1, -1, FAKE, 1, 1, FAKE, 1, 1, 1) == rs.INVALID_SIZE
    assert rs.call(g, handle, rs.FILL_LOWER, 2, 1, FAKE, 2, 1, FAKE, 1, 1, 1) == rs.INVALID_SIZE
    assert rs.call(g, handle, rs.FILL_LOWER, 1, 1, NULL, 1, 1, FAKE, 1, 1, 1) == rs.INVALID_POINTER
    assert rs.call(g, handle, rs.FILL_LOWER, 1, 1, FAKE, 1, 1, NULL, 1, 1, 1) == rs.INVALID_POINTER
    assert rs.call(g, handle, rs.FILL_LOWER, 1, 1, FAKE, 1, 1, FAKE, 1, 1, 0) == rs.SUCCESS
    v = f"rocsolver_{p}posv_strided_batched"
    assert rs.call(v, handle, rs.FILL_LOWER, 1, 1, FAKE, 1, 1, FAKE, 1, 1, NULL, 1) \
        == rs.INVALID_POINTER
    assert rs.call(v, handle, rs.FILL_LOWER, 1, 1, FAKE, 1, 1, FAKE, 1, 1, NULL, 0) == rs.SUCCESS


@pytest.mark.parametrize("p", ["s", "d", "c", "z"])
def test_getri_bad_args(handle, p):
    """clients/include/testing_getri.hpp:15-88 and testing_getri_outofplace.hpp bad-arg
    order: handle, sizes (n, lda, ldc, bc), then pointers (A, C, ipiv unless npvt, info)."""
    f = f"rocsolver_{p}getri_strided_batched"
    ok = dict(n=1, A=FAKE, lda=1, sA=1, ipiv=FAKE, sP=1, info=FAKE, bc=1)

    def c(h=handle, **kw):
        a = dict(ok, **kw)
        return rs.call(f, h, a["n"], a["A"], a["lda"], a["sA"], a["ipiv"], a["sP"], a["info"],
                       a["bc"])
    assert c(h=None) == rs.INVALID_HANDLE
    assert c(n=-1) == rs.INVALID_SIZE
    assert c(n=2, lda=1) == rs.INVALID_SIZE
    assert c(bc=-1) == rs.INVALID_SIZE
    assert c(n=-1, A=NULL) == rs.INVALID_SIZE
    for k in ("A", "ipiv", "info"):
        assert c(**{k: NULL}) == rs.INVALID_POINTER, k
    assert c(bc=0, info=NULL) == rs.SUCCESS
    assert rs.call(f"rocsolver_{p}getri_npvt_strided_batched", handle, 1, FAKE, 1, 1, NULL, 1) \
        == rs.INVALID_POINTER
    g = f"rocsolver_{p}getri_outofplace_strided_batched"
    # n, A, lda, sA, ipiv, sP, C, ldc, sC, info, bc
    assert rs.call(g, handle, 2, FAKE, 2, 4, FAKE, 2, FAKE, 1, 4, FAKE, 1) == rs.INVALID_SIZE
    assert rs.call(g, handle, 1, FAKE, 1, 1, FAKE, 1, NULL, 1, 1, FAKE, 1) == rs.INVALID_POINTER
    assert rs.call(g, handle, 1, FAKE, 1, 1, NULL, 1, FAKE, 1, 1, FAKE, 1) == rs.INVALID_POINTER
    assert rs.call(f"rocsolver_{p}getri_npvt_outofplace_strided_batched", handle, 1, FAKE, 1, 1,
                   FAKE, 1, 1, NULL, 1) == rs.INVALID_POINTER
    # in-place getri of an order too large for the on-chip inverse reports its workspace
    # (n*n elements per member) to a size query
    sz = ctypes.c_size_t()
    assert rs.call("rocblas_start_device_memory_size_query", handle) == rs.SUCCESS
    assert c(n=200, lda=200, sA=40000, sP=200, bc=10) == rs.SIZE_INCREASED
    assert rs.call("rocblas_stop_device_memory_size_query", handle, ctypes.byref(sz)) \
        == rs.SUCCESS
    assert sz.value >= 200 * 200 * 10 * {"s": 4, "d": 8, "c": 8, "z": 16}[p]


@pytest.mark.parametrize("p", ["s", "d", "c", "z"])
def test_gesv_outofplace_bad_args(handle, p):
    """clients/include/testing_gesv_outofplace.hpp:15-90 bad-arg order."""
    f = f"rocsolver_{p}gesv_outofplace"
    ok = dict(n=1, r=1, A=FAKE, lda=1, ipiv=FAKE, B=FAKE, ldb=1, X=FAKE, ldx=1, info=FAKE)

    def c(h=handle, **kw):
        a = dict(ok, **kw)
        return rs.call(f, h, a["n"], a["r"], a["A"], a["lda"], a["ipiv"], a["B"], a["ldb"],
                       a["X"], a["ldx"], a["info"])
    assert c(h=None) == rs.INVALID_HANDLE
    assert c(n=-1) == rs.INVALID_SIZE
    assert c(r=-1) == rs.INVALID_SIZE
    assert c(n=2, lda=1, ldb=2, ldx=2) == rs.INVALID_SIZE
    assert c(n=2, lda=2, ldb=2, ldx=1) == rs.INVALID_SIZE
    for k in ("A", "ipiv", "B", "X", "info"):
        assert c(**{k: NULL}) == rs.INVALID_POINTER, k


def test_memory_model_defaults_and_query(handle):
    """clients/gtest/memory_model_gtest.cpp:54-120: managed by default, 32 MiB nominal,
    a size query reports without computing and returns the size on stop."""
    sz = ctypes.c_size_t()
    assert rs.call("rocblas_is_managing_device_memory", handle) == 1
    rs.call("rocblas_get_device_memory_size", handle, ctypes.byref(sz))
    assert sz.value == 32 * 1024 * 1024
    assert rs.call("rocblas_start_device_memory_size_query", handle) == rs.SUCCESS
    assert rs.call("rocblas_is_device_memory_size_query", handle) == 1
    # getrf needs no workspace: the query is answered without launching anything
    st = rs.call("rocsolver_dgetrf_strided_batched", handle, 64, 64, FAKE, 64, 4096, FAKE, 64,
                 FAKE, 8)
    assert st == rs.SIZE_UNCHANGED
    # size errors still come first during a query; pointer errors do not
    st = rs.call("rocsolver_dgetrf_strided_batched", handle, -1, 64, FAKE, 64, 4096, FAKE, 64,
                 FAKE, 8)
    assert st == rs.INVALID_SIZE
    st = rs.call("rocsolver_dgetrf_strided_batched", handle, 64, 64, NULL, 64, 4096, NULL, 64,
                 NULL, 8)
    assert st == rs.SIZE_UNCHANGED
    assert rs.call("rocblas_stop_device_memory_size_query", handle, ctypes.byref(sz)) \
        == rs.SUCCESS
    assert sz.value == 0
    assert rs.call("rocblas_is_device_memory_size_query", handle) == 0
    assert rs.call("rocblas_stop_device_memory_size_query", handle, ctypes.byref(sz)) \
        == rs.SIZE_QUERY_MISMATCH


def test_memory_model_user_fixed(monkeypatch):
    monkeypatch.setenv("ROCBLAS_DEVICE_MEMORY_SIZE", "2000000")
    h = rs.Handle()
    try:
        sz = ctypes.c_size_t()
        assert rs.call("rocblas_is_managing_device_memory", h.value) == 0
        rs.call("rocblas_get_device_memory_size", h.value, ctypes.byref(sz))
        assert sz.value == 2000000
    finally:
        h.close()


def test_stream_roundtrip(handle):
    s = ctypes.c_void_p()
    assert rs.call("rocblas_set_stream", handle, ctypes.c_void_p(0x1234)) == rs.SUCCESS
    assert rs.call("rocblas_get_stream", handle, ctypes.byref(s)) == rs.SUCCESS
    assert s.value == 0x1234
    assert rs.call("rocblas_set_stream", handle, None) == rs.SUCCESS
