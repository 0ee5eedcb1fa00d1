"""GPU parity tests for the inverse from the LU factors (rocsolver_{s,d}getri, _npvt,
_outofplace, _npvt_outofplace, in their plain, _batched and _strided_batched forms) and for
rocsolver_{s,d}gesv_outofplace, through the C ABI against the golden LAPACK dgetri outputs
and the oracle.

Acceptance rules are the reference's (clients/include/testing_getri.hpp:209-233: info exact,
inverse within n*eps in the F-norm where info = 0; testing_gesv_outofplace.hpp:236-260:
solution within n*eps where info = 0), plus ||A inv(A) - I|| for uniform inputs."""
import os

import numpy as np
import pytest

import oracle
import rocsolver_b200 as rs
from tests.gpu_util import GpuHandle, dev, host, prefix, ptr, ptr_array
from tests.norms import eps_of, norm_error, solve_backward_error
from tests.refcases import from_colmajor, to_colmajor, uniform_general

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "lapack_golden.npz"))


@pytest.fixture(scope="module")
def handle():
    h = GpuHandle()
    yield h.value
    h.close()


def oracle_lu(A, pivot=True):
    bc, n, _ = A.shape
    flat = to_colmajor(A)
    ipiv = np.zeros(bc * max(n, 1), np.int32)
    info = np.zeros(bc, np.int32)
    oracle.getrf(n, n, flat, n, n * n, ipiv, max(n, 1), info, bc, pivot=pivot,
                 nthreads=oracle.nthreads_default())
    return from_colmajor(flat, bc, n, n, n, n * n), ipiv.reshape(bc, max(n, 1))[:, :n], info


def oracle_inv(LU, ipiv, pivot=True):
    bc, n, _ = LU.shape
    flat = to_colmajor(LU)
    info = np.zeros(bc, np.int32)
    oracle.getri(n, flat, n, n * n, ipiv.astype(np.int32).reshape(-1).copy(), n, info, bc,
                 pivot=pivot, nthreads=oracle.nthreads_default())
    return from_colmajor(flat, bc, n, n, n, n * n), info


def gpu_getri(handle, LU, ipiv, form="strided", pivot=True, lda=None, outofplace=False,
              ldc=None):
    """Run one getri form; returns (inverse, info, factors after the call)."""
    bc, n, _ = LU.shape
    lda = n if lda is None else lda
    ldc = n if ldc is None else ldc
    p = prefix(LU.dtype)
    dA = dev(to_colmajor(LU, lda))
    dP = dev(np.ascontiguousarray(ipiv, np.int32).reshape(-1)) if pivot else None
    dI = dev(np.full(bc, -9, np.int32))
    dC = dev(np.full(max(ldc * n * bc, 1), np.nan, LU.dtype)) if outofplace else None
    name = f"rocsolver_{p}getri" + ("_npvt" if not pivot else "") \
        + ("_outofplace" if outofplace else "")
    piv_args = [ptr(dP)] if pivot else []
    if form == "plain":
        assert bc == 1
        args = [n, ptr(dA), lda] + piv_args + ([ptr(dC), ldc] if outofplace else []) + [ptr(dI)]
        st = rs.call(name, handle, *args)
    elif form == "batched":
        aA = ptr_array(dA, bc, lda * n)
        aC = ptr_array(dC, bc, ldc * n) if outofplace else None
        args = [n, ptr(aA), lda] + (piv_args + [n] if pivot else []) \
            + ([ptr(aC), ldc] if outofplace else []) + [ptr(dI), bc]
        st = rs.call(name + "_batched", handle, *args)
        host(dI)
    else:
        args = [n, ptr(dA), lda, lda * n] + (piv_args + [n] if pivot else []) \
            + ([ptr(dC), ldc, ldc * n] if outofplace else []) + [ptr(dI), bc]
        st = rs.call(name + "_strided_batched", handle, *args)
    assert st == rs.SUCCESS, rs.STATUS_NAMES[st]
    A_after = from_colmajor(host(dA), bc, n, n, lda, lda * n)
    inv = from_colmajor(host(dC), bc, n, n, ldc, ldc * n) if outofplace else A_after
    return inv, host(dI), A_after


@pytest.mark.parametrize("n,singular", [(32, 0), (50, 1), (70, 0), (100, 1)])
@pytest.mark.parametrize("form", ["strided", "batched"])
def test_getri_reference_suite(handle, n, singular, form):
    key = f"getri_ref_n{n}_s{singular}"
    LU, ipiv = GOLD[key + "_LU"], GOLD[key + "_ipiv"]
    inv, info, _ = gpu_getri(handle, LU, ipiv, form=form)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    for b in range(3):
        if info[b] == 0:
            assert norm_error("F", GOLD[key + "_inv"][b], inv[b]) <= n * eps_of(np.float64)
        else:  # LAPACK dgetri leaves the factors of a singular member untouched
            np.testing.assert_array_equal(inv[b], LU[b])


@pytest.mark.parametrize("n,singular", [(32, 0), (50, 1), (100, 1)])
def test_getri_outofplace_reference_suite(handle, n, singular):
    key = f"getri_ref_n{n}_s{singular}"
    LU, ipiv = GOLD[key + "_LU"], GOLD[key + "_ipiv"]
    inv, info, after = gpu_getri(handle, LU, ipiv, outofplace=True, ldc=n + 5)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    np.testing.assert_array_equal(after, LU)  # A is not modified
    for b in range(3):
        if info[b] == 0:
            assert norm_error("F", GOLD[key + "_inv"][b], inv[b]) <= n * eps_of(np.float64)


@pytest.mark.parametrize("n", [1, 2, 7, 31, 32, 33, 64, 100, 256, 300])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("outofplace", [False, True])
def test_getri_vs_oracle(handle, n, dtype, outofplace):
    A = uniform_general(n, n, 3, seed=4000 + n).astype(dtype)
    LU, ipiv, finfo = oracle_lu(A)
    assert not finfo.any()
    oinv, oinfo = oracle_inv(LU, ipiv)
    inv, info, _ = gpu_getri(handle, LU, ipiv, outofplace=outofplace, lda=n + 2,
                             form="batched" if n == 33 else "strided")
    np.testing.assert_array_equal(info, oinfo)
    eps = eps_of(dtype)
    for b in range(3):
        # two inverses of the same factors differ by ~cond(A) eps; the residual is the check
        r = np.abs(A[b].astype(np.float64) @ inv[b].astype(np.float64) - np.eye(n)).max()
        kappa = np.linalg.cond(A[b].astype(np.float64), np.inf)
        assert r <= 10 * n * eps * max(1.0, kappa), (b, r)
        assert norm_error("F", oinv[b], inv[b]) <= 10 * n * eps * max(1.0, kappa)


@pytest.mark.parametrize("n", [5, 32, 64, 130])
@pytest.mark.parametrize("outofplace", [False, True])
def test_getri_npvt(handle, n, outofplace):
    A = uniform_general(n, n, 2, seed=4100 + n) + n * np.eye(n)[None]
    LU, _, finfo = oracle_lu(A, pivot=False)
    assert not finfo.any()
    oinv, oinfo = oracle_inv(LU, np.zeros((2, n), np.int32), pivot=False)
    inv, info, _ = gpu_getri(handle, LU, None, pivot=False, outofplace=outofplace)
    np.testing.assert_array_equal(info, oinfo)
    for b in range(2):
        assert norm_error("F", oinv[b], inv[b]) <= 10 * n * eps_of(np.float64)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_getri_plain_forms_and_singular(handle, dtype):
    """rocsolver_{s,d}getri and getri_outofplace on one matrix; a zero U(i,i) gives info =
    i + 1 and leaves the factors in place."""
    n = 40
    A = uniform_general(n, n, 1, seed=77).astype(dtype)
    LU, ipiv, _ = oracle_lu(A)
    oinv, _ = oracle_inv(LU, ipiv)
    for oop in (False, True):
        inv, info, _ = gpu_getri(handle, LU, ipiv, form="plain", outofplace=oop)
        assert info[0] == 0
        assert norm_error("F", oinv[0], inv[0]) <= 100 * n * eps_of(dtype)
    S = LU.copy()
    S[0, 17, 17] = 0
    S[0, 30, 30] = 0
    inv, info, after = gpu_getri(handle, S, ipiv, form="plain")
    assert info[0] == 18
    np.testing.assert_array_equal(after, S)


@pytest.mark.parametrize("n", [1, 8, 32, 33, 100, 256])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_gesv_outofplace(handle, n, dtype):
    """X = A^{-1} B, B unchanged, A overwritten by its factors; pivots and info exactly the
    oracle's; a singular A gives info > 0 (X then keeps the copy of B)."""
    p = prefix(dtype)
    eps = eps_of(dtype)
    nrhs = 3
    for singular in (False, True):
        A = uniform_general(n, n, 1, seed=4200 + n).astype(dtype)
        if singular:
            A[0, :, n // 2] = 0
        B = uniform_general(n, nrhs, 1, seed=4300 + n).astype(dtype)
        lda, ldb, ldx = n + 1, n + 2, n + 3
        dA, dB = dev(to_colmajor(A, lda)), dev(to_colmajor(B, ldb))
        dX = dev(np.full(ldx * nrhs, np.nan, dtype))
        dP, dI = dev(np.zeros(n, np.int32)), dev(np.full(1, -1, np.int32))
        st = rs.call(f"rocsolver_{p}gesv_outofplace", handle, n, nrhs, ptr(dA), lda, ptr(dP),
                     ptr(dB), ldb, ptr(dX), ldx, ptr(dI))
        assert st == rs.SUCCESS
        Bafter = from_colmajor(host(dB), 1, n, nrhs, ldb, ldb * nrhs)[0]
        np.testing.assert_array_equal(Bafter, B[0])
        oA, oB = to_colmajor(A), to_colmajor(B)
        oP, oI = np.zeros(n, np.int32), np.zeros(1, np.int32)
        oracle.gesv(n, nrhs, oA, n, n * n, oP, n, oB, n, n * nrhs, oI, 1)
        info = host(dI)
        assert info[0] == oI[0]
        assert (info[0] > 0) == singular
        X = from_colmajor(host(dX), 1, n, nrhs, ldx, ldx * nrhs)[0]
        if not singular:
            np.testing.assert_array_equal(host(dP), oP)
            assert solve_backward_error(A[0].astype(np.float64), X.astype(np.float64),
                                        B[0].astype(np.float64)) < 10 * n * eps
        else:
            np.testing.assert_array_equal(X, B[0])
