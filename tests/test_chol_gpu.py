"""GPU parity tests for potrf / potrs / posv through the C ABI against the oracle and the
golden LAPACK fixtures (clients/include/testing_potf2_potrf.hpp:186-210,450: info exact,
leading nn x nn triangle F-norm error <= n*eps; testing_potrs.hpp:210-220,425 and
testing_posv.hpp: solution inf-norm error <= n*eps)."""
import os

import numpy as np
import pytest

import oracle
import rocsolver_b200 as rs
from tests.gpu_util import GpuHandle, dev, host, prefix, ptr, ptr_array
from tests.norms import eps_of, norm_error, norm_error_lower, norm_error_upper, \
    solve_backward_error
from tests.refcases import from_colmajor, ref_potrf_input, spd_gram, to_colmajor

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "lapack_golden.npz"))


@pytest.fixture(scope="module")
def handle():
    h = GpuHandle()
    yield h.value
    h.close()


def gpu_potrf(handle, A, lower, lda=None, batched=False):
    bc, n, _ = A.shape
    lda = n if lda is None else lda
    dA = dev(to_colmajor(A, lda))
    dI = dev(np.full(bc, -5, np.int32))
    p = prefix(A.dtype)
    uplo = rs.FILL_LOWER if lower else rs.FILL_UPPER
    if batched:
        arr = ptr_array(dA, bc, lda * n)  # keep alive until the kernel has run
        st = rs.call(f"rocsolver_{p}potrf_batched", handle, uplo, n, ptr(arr), lda, ptr(dI), bc)
        host(dI)
    else:
        st = rs.call(f"rocsolver_{p}potrf_strided_batched", handle, uplo, n, ptr(dA), lda,
                     lda * n, ptr(dI), bc)
    assert st == rs.SUCCESS
    raw = host(dA)
    return from_colmajor(raw, bc, n, n, lda, lda * n), host(dI), raw


def oracle_potrf(A, lower):
    bc, n, _ = A.shape
    flat = to_colmajor(A)
    info = np.zeros(bc, np.int32)
    oracle.potrf(not lower, n, flat, n, n * n, info, bc, nthreads=oracle.nthreads_default())
    return from_colmajor(flat, bc, n, n, n, n * n), info


def check_potrf(A, C, info, lower, untouched_other=True):
    bc, n, _ = A.shape
    oC, oinfo = oracle_potrf(A, lower)
    np.testing.assert_array_equal(info, oinfo)
    f = norm_error_lower if lower else norm_error_upper
    eps = eps_of(A.dtype)
    for b in range(bc):
        nn = n if info[b] == 0 else info[b]
        assert f("F", oC[b][:nn, :nn], C[b][:nn, :nn]) <= n * eps * 4
        if untouched_other:
            strict = np.triu(np.ones((n, n), bool), 1) if lower else np.tril(np.ones((n, n), bool), -1)
            np.testing.assert_array_equal(C[b][strict], A[b][strict])


@pytest.mark.parametrize("n", [10, 20, 50, 70])
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("singular", [False, True])
def test_potrf_reference_suite(handle, n, lower, singular):
    A = ref_potrf_input(n, 3, singular)
    C, info, _ = gpu_potrf(handle, A, lower)
    key = f"potrf_ref_n{n}_L{int(lower)}_s{int(singular)}"
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    f = norm_error_lower if lower else norm_error_upper
    for b in range(3):
        nn = n if info[b] == 0 else info[b]
        assert f("F", GOLD[key + "_C"][b][:nn, :nn], C[b][:nn, :nn]) <= n * eps_of(np.float64)
    check_potrf(A, C, info, lower)


@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 63, 64, 65, 100, 200, 256, 300, 512, 700])
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_potrf_spd(handle, n, lower, dtype):
    A = spd_gram(n, 3, seed=n + 17).astype(dtype)
    A[1, n // 2, n // 2] = -1.0  # not positive definite from order n//2+1 on (or earlier)
    C, info, _ = gpu_potrf(handle, A, lower, lda=n + (n % 3), batched=(n == 33))
    check_potrf(A, C, info, lower)


def gpu_potrs(handle, C, B, lower, batched=False):
    bc, n, _ = C.shape
    nrhs = B.shape[2]
    dA = dev(to_colmajor(C))
    dB = dev(to_colmajor(B))
    p = prefix(C.dtype)
    uplo = rs.FILL_LOWER if lower else rs.FILL_UPPER
    if batched:
        aA, aB = ptr_array(dA, bc, n * n), ptr_array(dB, bc, n * nrhs)
        st = rs.call(f"rocsolver_{p}potrs_batched", handle, uplo, n, nrhs, ptr(aA), n, ptr(aB),
                     n, bc)
        host(dB)
    else:
        st = rs.call(f"rocsolver_{p}potrs_strided_batched", handle, uplo, n, nrhs, ptr(dA), n,
                     n * n, ptr(dB), n, n * nrhs, bc)
    assert st == rs.SUCCESS
    return from_colmajor(host(dB), bc, n, nrhs, n, n * nrhs)


@pytest.mark.parametrize("n", [1, 2, 31, 33, 64, 65])
@pytest.mark.parametrize("lower", [True, False])
def test_potrs_golden(handle, n, lower):
    key = f"potrs_spd_n{n}_L{int(lower)}"
    B = np.random.default_rng(300 + n).standard_normal((4, n, 4))
    X = gpu_potrs(handle, GOLD[key + "_C"], B, lower, batched=(n == 31))
    for b in range(4):
        assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * eps_of(np.float64) * 4


@pytest.mark.parametrize("n", [8, 64, 100, 256])
@pytest.mark.parametrize("nrhs", [1, 4, 9])
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_posv_vs_oracle(handle, n, nrhs, lower, dtype):
    A = spd_gram(n, 3, seed=n * 3 + nrhs).astype(dtype)
    A[2, 3, 3] = -5.0  # failing member keeps its B
    B = np.random.default_rng(n + nrhs).standard_normal((3, n, nrhs)).astype(dtype)
    dA = dev(to_colmajor(A))
    dB = dev(to_colmajor(B))
    dI = dev(np.full(3, -1, np.int32))
    p = prefix(dtype)
    uplo = rs.FILL_LOWER if lower else rs.FILL_UPPER
    st = rs.call(f"rocsolver_{p}posv_strided_batched", handle, uplo, n, nrhs, ptr(dA), n, n * n,
                 ptr(dB), n, n * nrhs, ptr(dI), 3)
    assert st == rs.SUCCESS
    X = from_colmajor(host(dB), 3, n, nrhs, n, n * nrhs)
    info = host(dI)
    oA, oB, oI = to_colmajor(A), to_colmajor(B), np.zeros(3, np.int32)
    oracle.posv(not lower, n, nrhs, oA, n, n * n, oB, n, n * nrhs, oI, 3)
    np.testing.assert_array_equal(info, oI)
    eps = eps_of(dtype)
    for b in range(3):
        if info[b] != 0:
            np.testing.assert_array_equal(X[b], B[b])
        else:
            be = solve_backward_error(A[b].astype(np.float64), X[b].astype(np.float64),
                                      B[b].astype(np.float64))
            assert be < 10 * n * eps


def test_config_potrf_n64_bc20000(handle):
    """dpotrf + dpotrs, n=64, batch=20000, nrhs=4, A = G G' + n I: info bit-exact against
    the oracle for every member; factor and solution within tolerance on a sample."""
    n, bc = 64, 20000
    rng = np.random.default_rng(1)
    G = rng.standard_normal((bc, n, n))
    A = G @ G.transpose(0, 2, 1) + n * np.eye(n)[None]
    B = rng.standard_normal((bc, n, 4))
    C, info, _ = gpu_potrf(handle, A, True)
    oC, oinfo = oracle_potrf(A, True)
    np.testing.assert_array_equal(info, oinfo)
    assert not info.any()
    for b in range(0, bc, 97):
        assert norm_error_lower("F", oC[b], C[b]) <= n * eps_of(np.float64)
    X = gpu_potrs(handle, C, B, True)
    for b in range(0, bc, 97):
        be = solve_backward_error(A[b], X[b], B[b])
        assert be < 10 * n * eps_of(np.float64)
