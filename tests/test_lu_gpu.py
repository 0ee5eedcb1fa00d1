"""GPU parity tests for getrf / getrs / gesv through the C ABI, against the oracle (which
tests/test_oracle.py pins to host LAPACK) and the golden LAPACK fixtures.

Acceptance rules are the reference's (clients/include/testing_getf2_getrf.hpp:233-259,504:
ipiv and info exact, factor F-norm error <= min(m,n)*eps; testing_getrs.hpp:219-229,462 and
testing_gesv.hpp:229-247,506: solution inf-norm error <= n*eps), plus the backward errors
of the benchmarked configurations: ||PA - LU||_F / (n ||A||_F eps) < 10 and
||AX - B|| / (||A|| ||X|| + ||B||) reported per member."""
import os

import numpy as np
import pytest

import oracle
import rocsolver_b200 as rs
from tests.gpu_util import GpuHandle, dev, host, prefix, ptr, ptr_array
from tests.norms import eps_of, lu_backward_error, norm_error, solve_backward_error
from tests.refcases import (from_colmajor, ref_gesv_input, ref_getrf_input, ref_getrs_input,
                            to_colmajor, uniform_general)

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "lapack_golden.npz"))


@pytest.fixture(scope="module")
def handle():
    h = GpuHandle()
    yield h.value
    h.close()


def gpu_getrf(handle, A, lda=None, stride=None, pivot=True, batched=False, strideP=None):
    bc, m, n = A.shape
    lda = m if lda is None else lda
    stride = lda * n if stride is None else stride
    mn = max(min(m, n), 1)
    strideP = mn if strideP is None else strideP
    flat = to_colmajor(A, lda, stride)
    dA = dev(flat)
    dP = dev(np.full(max(bc * strideP, 1), -7, np.int32))
    dI = dev(np.full(bc, -7, np.int32))
    p = prefix(A.dtype)
    if batched:
        arr = ptr_array(dA, bc, stride)
        if pivot:
            st = rs.call(f"rocsolver_{p}getrf_batched", handle, m, n, ptr(arr), lda, ptr(dP),
                         strideP, ptr(dI), bc)
        else:
            st = rs.call(f"rocsolver_{p}getrf_npvt_batched", handle, m, n, ptr(arr), lda,
                         ptr(dI), bc)
        host(dI)
    elif pivot:
        st = rs.call(f"rocsolver_{p}getrf_strided_batched", handle, m, n, ptr(dA), lda, stride,
                     ptr(dP), strideP, ptr(dI), bc)
    else:
        st = rs.call(f"rocsolver_{p}getrf_npvt_strided_batched", handle, m, n, ptr(dA), lda,
                     stride, ptr(dI), bc)
    assert st == rs.SUCCESS, rs.STATUS_NAMES[st]
    out = host(dA)
    LU = from_colmajor(out, bc, m, n, lda, stride)
    ipiv = host(dP)
    info = host(dI)
    return LU, ipiv, info, out


def oracle_getrf(A, pivot=True):
    bc, m, n = A.shape
    flat = to_colmajor(A)
    mn = max(min(m, n), 1)
    ipiv = np.zeros(bc * mn, np.int32)
    info = np.zeros(bc, np.int32)
    oracle.getrf(m, n, flat, m, m * n, ipiv, mn, info, bc, pivot=pivot,
                 nthreads=oracle.nthreads_default())
    return from_colmajor(flat, bc, m, n, m, m * n), ipiv.reshape(bc, mn)[:, :min(m, n)], info


def check_getrf(A, LU, ipiv_flat, info, pivot=True, strideP=None):
    bc, m, n = A.shape
    mn = min(m, n)
    oLU, oipiv, oinfo = oracle_getrf(A, pivot)
    np.testing.assert_array_equal(info, oinfo)
    if pivot and mn > 0:
        sp = strideP if strideP is not None else mn
        gp = ipiv_flat[: bc * sp].reshape(bc, sp)[:, :mn]
        np.testing.assert_array_equal(gp, oipiv)
    eps = eps_of(A.dtype)
    for b in range(bc):
        err = norm_error("F", oLU[b], LU[b])
        assert err <= max(mn, 1) * eps * 4, (b, err / eps)


SIZES_REF = [(32, 16), (32, 20), (32, 40), (32, 100), (50, 16), (50, 20), (50, 40), (50, 100),
             (70, 16), (70, 20), (70, 40), (70, 100)]


@pytest.mark.parametrize("m,n", SIZES_REF)
@pytest.mark.parametrize("singular", [False, True])
def test_getrf_reference_suite_d(handle, m, n, singular):
    A = ref_getrf_input(m, n, m, 3, singular)
    LU, ipiv, info, _ = gpu_getrf(handle, A)
    key = f"getrf_ref_m{m}_n{n}_s{int(singular)}"
    mn = min(m, n)
    np.testing.assert_array_equal(ipiv.reshape(3, mn), GOLD[key + "_ipiv"])
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    for b in range(3):
        assert norm_error("F", GOLD[key + "_LU"][b], LU[b]) <= mn * eps_of(np.float64)
    check_getrf(A, LU, ipiv, info)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 9, 16, 17, 31, 32, 33, 63, 64, 65, 100, 128, 129,
                               255, 256, 257, 300, 512])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_getrf_uniform_square(handle, n, dtype):
    A = uniform_general(n, n, 5, seed=1000 + n).astype(dtype)
    LU, ipiv, info, _ = gpu_getrf(handle, A)
    check_getrf(A, LU, ipiv, info)
    if dtype == np.float64:
        for b in range(A.shape[0]):
            be = lu_backward_error(A[b], LU[b], ipiv.reshape(5, n)[b])
            assert be / (n * eps_of(dtype)) < 10


@pytest.mark.parametrize("n", [16, 33, 64, 100, 128, 200, 256, 300, 512, 1024])
def test_sgetrf_tf32(handle, n):
    """rocsolver_sgetrf_tf32_strided_batched (split-TF32 tensor-core trailing updates, the
    factorisation of dsgesv): info as the oracle's FP32 LU, FP32-level backward error
    ||PA - LU||_F / (n ||A||_F eps32) < 10 with the returned pivots, and up to n = 512 the
    oracle's pivots except where the different rounding flips a near tie (< 2 % of them;
    at n = 1024 one early flip changes every later pivot, so only the backward error and
    info are compared)."""
    bc = 3
    A = uniform_general(n, n, bc, seed=4000 + n).astype(np.float32)
    dA = dev(to_colmajor(A))
    dP = dev(np.full(bc * n, -7, np.int32))
    dI = dev(np.full(bc, -7, np.int32))
    st = rs.call("rocsolver_sgetrf_tf32_strided_batched", handle, n, n, ptr(dA), n, n * n,
                 ptr(dP), n, ptr(dI), bc)
    assert st == rs.SUCCESS, rs.STATUS_NAMES[st]
    LU = from_colmajor(host(dA), bc, n, n, n, n * n)
    ipiv, info = host(dP).reshape(bc, n), host(dI)
    _, oipiv, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(info, oinfo)
    for b in range(bc):
        be = lu_backward_error(A[b].astype(np.float64), LU[b].astype(np.float64), ipiv[b])
        assert be / (n * eps_of(np.float32)) < 10, (b, be)
    if n <= 512:
        assert (ipiv != oipiv).mean() < 0.02


def test_sgetrf_tf32_argument_checks(handle):
    """Same checks and quick returns as sgetrf (roclapack_getrf_strided_batched.cpp:8-84)."""
    dI = dev(np.full(2, -7, np.int32))
    f = "rocsolver_sgetrf_tf32_strided_batched"
    assert rs.call(f, None, 4, 4, None, 4, 16, None, 4, ptr(dI), 2) == rs.INVALID_HANDLE
    assert rs.call(f, handle, -1, 4, None, 4, 16, None, 4, ptr(dI), 2) == rs.INVALID_SIZE
    assert rs.call(f, handle, 4, 4, None, 3, 16, None, 4, ptr(dI), 2) == rs.INVALID_SIZE
    assert rs.call(f, handle, 4, 4, None, 4, 16, None, 4, ptr(dI), 2) == rs.INVALID_POINTER
    assert rs.call(f, handle, 0, 4, None, 1, 4, None, 4, ptr(dI), 2) == rs.SUCCESS
    np.testing.assert_array_equal(host(dI), [0, 0])


@pytest.mark.parametrize("m,n", [(1, 5), (5, 1), (7, 3), (3, 7), (31, 33), (33, 31), (64, 16),
                                 (16, 64), (200, 40), (40, 200), (513, 60), (192, 520),
                                 (640, 64), (1000, 45)])
def test_getrf_rectangular(handle, m, n):
    A = uniform_general(m, n, 2, seed=m * 1000 + n)
    LU, ipiv, info, _ = gpu_getrf(handle, A)
    check_getrf(A, LU, ipiv, info)


def test_getrf_padding_untouched(handle):
    """lda > m and strideA > lda*n: padding (NaN sentinels) must be unchanged."""
    m = n = 40
    A = uniform_general(m, n, 3, seed=5)
    lda, stride = 45, 45 * 40 + 37
    LU, ipiv, info, raw = gpu_getrf(handle, A, lda=lda, stride=stride, strideP=50)
    for b in range(3):
        blk = raw[b * stride: b * stride + lda * n].reshape(n, lda)
        assert np.all(np.isnan(blk[:, m:]))
        if b < 2:
            assert np.all(np.isnan(raw[b * stride + lda * n:(b + 1) * stride]))
    check_getrf(A, LU, ipiv, info, strideP=50)
    np.testing.assert_array_equal(ipiv.reshape(3, 50)[:, 40:], -7)


@pytest.mark.parametrize("n", [20, 32, 100])
def test_getrf_batched_pointer_array(handle, n):
    A = uniform_general(n, n, 4, seed=77 + n)
    LU, ipiv, info, _ = gpu_getrf(handle, A, batched=True)
    check_getrf(A, LU, ipiv, info)


@pytest.mark.parametrize("n", [8, 32, 50, 256])
def test_getrf_npvt(handle, n):
    A = uniform_general(n, n, 3, seed=9 + n) + 2.0 * n * np.eye(n)[None]
    LU, _, info, _ = gpu_getrf(handle, A, pivot=False)
    check_getrf(A, LU, None, info, pivot=False)


@pytest.mark.parametrize("n", [32, 256])
def test_getrf_nan_and_zero_columns(handle, n):
    """A NaN below the diagonal never becomes the pivot (LAPACK idamax rule); an exactly
    zero column gives info = its 1-based index and no interchange."""
    A = uniform_general(n, n, 4, seed=3)
    A[1, :, 7] = 0.0              # whole column 7 zero -> info = 8
    A[2, n // 2, 0] = np.nan      # NaN below the first pivot candidate: never chosen
    A[3, 0, 0] = np.nan           # NaN on the first candidate row: it stays the pivot
    LU, ipiv, info, _ = gpu_getrf(handle, A)
    oLU, oipiv, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(info, oinfo)
    np.testing.assert_array_equal(ipiv.reshape(4, n), oipiv)
    assert info[1] == 8
    assert ipiv.reshape(4, n)[3, 0] == 1


def test_getrf_quick_returns(handle):
    dI = dev(np.full(4, 9, np.int32))
    st = rs.call("rocsolver_dgetrf_strided_batched", handle, 0, 5, None, 1, 5, None, 5,
                 ptr(dI), 4)
    assert st == rs.SUCCESS
    np.testing.assert_array_equal(host(dI), 0)


# ------------------------------------------------------------------------------- getrs
def gpu_getrs(handle, trans, LU, ipiv, B, ldb=None, batched=False):
    bc, n, _ = LU.shape
    nrhs = B.shape[2]
    ldb = n if ldb is None else ldb
    dA = dev(to_colmajor(LU))
    dB = dev(to_colmajor(B, ldb))
    dP = dev(ipiv.astype(np.int32).reshape(-1))
    p = prefix(LU.dtype)
    op = rs.OP_T if trans else rs.OP_N
    if batched:
        aA = ptr_array(dA, bc, n * n)
        aB = ptr_array(dB, bc, ldb * nrhs)
        st = rs.call(f"rocsolver_{p}getrs_batched", handle, op, n, nrhs, ptr(aA), n, ptr(dP), n,
                     ptr(aB), ldb, bc)
        host(dB)
    else:
        st = rs.call(f"rocsolver_{p}getrs_strided_batched", handle, op, n, nrhs, ptr(dA), n,
                     n * n, ptr(dP), n, ptr(dB), ldb, ldb * nrhs, bc)
    assert st == rs.SUCCESS
    return from_colmajor(host(dB), bc, n, nrhs, ldb, ldb * nrhs)


@pytest.mark.parametrize("n", [20, 30, 50])
@pytest.mark.parametrize("nrhs", [10, 20, 30])
@pytest.mark.parametrize("trans", [0, 1])
def test_getrs_reference_suite(handle, n, nrhs, trans):
    key = f"getrs_ref_n{n}_r{nrhs}_t{trans}"
    _, B = ref_getrs_input(n, nrhs, 3)
    X = gpu_getrs(handle, trans, GOLD[key + "_LU"], GOLD[key + "_ipiv"], B)
    for b in range(3):
        assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * eps_of(np.float64)


@pytest.mark.parametrize("n", [1, 5, 16, 31, 32, 33, 64, 100, 256, 300])
@pytest.mark.parametrize("nrhs", [1, 3, 8])
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_getrs_vs_oracle(handle, n, nrhs, trans, dtype):
    A = uniform_general(n, n, 3, seed=n * 7 + nrhs).astype(dtype)
    B = uniform_general(n, nrhs, 3, seed=n * 11 + nrhs).astype(dtype)
    LU, ipiv, info = oracle_getrf(A)
    X = gpu_getrs(handle, trans, LU, ipiv, B, ldb=n + 3, batched=(n == 33))
    Bf = to_colmajor(B)
    oracle.getrs(trans, n, nrhs, to_colmajor(LU), n, n * n, ipiv.astype(np.int32).reshape(-1).copy(),
                 n, Bf, n, n * nrhs, 3)
    OX = from_colmajor(Bf, 3, n, nrhs, n, n * nrhs)
    eps = eps_of(dtype)
    for b in range(3):
        # the oracle solution carries cond(A)*eps error of its own; compare normwise
        assert norm_error("I", OX[b], X[b]) <= max(n, 1) * eps * 50
        opA = A[b].T if trans else A[b]
        be = solve_backward_error(opA.astype(np.float64), X[b].astype(np.float64),
                                  B[b].astype(np.float64))
        assert be < 10 * n * eps


# ------------------------------------------------------------------------------- gesv
def gpu_gesv(handle, A, B, batched=False):
    bc, n, _ = A.shape
    nrhs = B.shape[2]
    dA = dev(to_colmajor(A))
    dB = dev(to_colmajor(B))
    dP = dev(np.zeros(bc * n, np.int32))
    dI = dev(np.full(bc, -3, np.int32))
    p = prefix(A.dtype)
    if batched:
        aA, aB = ptr_array(dA, bc, n * n), ptr_array(dB, bc, n * nrhs)  # alive until run
        st = rs.call(f"rocsolver_{p}gesv_batched", handle, n, nrhs, ptr(aA), n, ptr(dP), n,
                     ptr(aB), n, ptr(dI), bc)
        host(dI)
    else:
        st = rs.call(f"rocsolver_{p}gesv_strided_batched", handle, n, nrhs, ptr(dA), n, n * n,
                     ptr(dP), n, ptr(dB), n, n * nrhs, ptr(dI), bc)
    assert st == rs.SUCCESS
    return (from_colmajor(host(dA), bc, n, n, n, n * n), host(dP).reshape(bc, n),
            from_colmajor(host(dB), bc, n, nrhs, n, n * nrhs), host(dI))


@pytest.mark.parametrize("n", [20, 35, 50])
@pytest.mark.parametrize("nrhs", [1, 10])
@pytest.mark.parametrize("singular", [False, True])
def test_gesv_reference_suite(handle, n, nrhs, singular):
    key = f"gesv_ref_n{n}_r{nrhs}_s{int(singular)}"
    A, B = ref_gesv_input(n, nrhs, 3, singular)
    LU, ipiv, X, info = gpu_gesv(handle, A, B)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    np.testing.assert_array_equal(ipiv, GOLD[key + "_ipiv"])
    for b in range(3):
        if info[b] == 0:
            assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * eps_of(np.float64)
        else:
            np.testing.assert_array_equal(X[b], B[b])


@pytest.mark.parametrize("n", [1, 7, 16, 32, 33, 64, 128, 256])
@pytest.mark.parametrize("nrhs", [1, 4])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_gesv_vs_oracle(handle, n, nrhs, dtype):
    A = uniform_general(n, n, 4, seed=n + 500).astype(dtype)
    B = uniform_general(n, nrhs, 4, seed=n + 600).astype(dtype)
    A[2, :, n // 2] = 0  # singular member: B must come back unchanged
    LU, ipiv, X, info = gpu_gesv(handle, A, B, batched=(n == 16))
    oA, oB = to_colmajor(A), to_colmajor(B)
    oP, oI = np.zeros(4 * n, np.int32), np.zeros(4, np.int32)
    oracle.gesv(n, nrhs, oA, n, n * n, oP, n, oB, n, n * nrhs, oI, 4)
    np.testing.assert_array_equal(info, oI)
    np.testing.assert_array_equal(ipiv, oP.reshape(4, n))
    eps = eps_of(dtype)
    for b in range(4):
        if info[b] != 0:
            np.testing.assert_array_equal(X[b], B[b])
        else:
            be = solve_backward_error(A[b].astype(np.float64), X[b].astype(np.float64),
                                      B[b].astype(np.float64))
            assert be < 10 * n * eps


# ------------------------------------------------------- benchmarked shapes at full size
def test_config_getrf_n32_bc1000(handle):
    """Plain dgetrf+dgetrs, n=32, lda=32, batch=1000, nrhs=1, uniform[-1,1] from seed 0:
    ipiv and info bit-exact against the oracle for every member, residual within the
    normwise tolerance."""
    rng = np.random.default_rng(0)
    A = rng.uniform(-1, 1, (1000, 32, 32))
    B = rng.uniform(-1, 1, (1000, 32, 1))
    LU, ipiv, info, _ = gpu_getrf(handle, A)
    oLU, oipiv, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(ipiv.reshape(1000, 32), oipiv)
    np.testing.assert_array_equal(info, oinfo)
    X = gpu_getrs(handle, 0, LU, ipiv.reshape(1000, 32), B)
    eps = eps_of(np.float64)
    worst_lu = max(lu_backward_error(A[b], LU[b], ipiv.reshape(1000, 32)[b]) for b in range(1000))
    assert worst_lu / (32 * eps) < 10
    for b in range(0, 1000, 10):
        r = A[b] @ X[b] - B[b]
        rel = np.abs(r).max() / (np.abs(A[b]).sum(1).max() * np.abs(X[b]).max() * 32 * eps)
        assert rel < 10


def test_config_getrf_n256_subset(handle):
    """Plain FP64 LU at n=256 (the mixed-precision comparator shape): ipiv/info exact
    against the oracle on 32 members, backward error < 10."""
    A = uniform_general(256, 256, 32, seed=42)
    LU, ipiv, info, _ = gpu_getrf(handle, A)
    check_getrf(A, LU, ipiv, info)
    for b in range(32):
        be = lu_backward_error(A[b], LU[b], ipiv.reshape(32, 256)[b])
        assert be / (256 * eps_of(np.float64)) < 10
