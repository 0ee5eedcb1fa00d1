"""GPU parity tests of the complex precisions (c = rocblas_float_complex, z =
rocblas_double_complex) through the C ABI: getrf (and npvt), getrs with N / T / C, gesv, potrf
and potrs (Hermitian, lower and upper), posv, in the plain, pointer-array and strided forms.
The checker is the complex oracle (tests/test_oracle_complex.py pins it to host LAPACK
zgetrf / zgetrs / zpotrf / zpotrs / zgesv) and the golden fixtures themselves.  Acceptance
rules are the reference's (clients/include/testing_getf2_getrf.hpp:233-259: ipiv and info
exact, factors within min(m,n)*eps in the F-norm; testing_getrs.hpp:219-229 and
testing_gesv.hpp:229-247: solutions within n*eps in the inf-norm; testing_potf2_potrf.hpp:
186-210: the referenced triangle within n*eps)."""
import os

import numpy as np
import pytest

import oracle
import rocsolver_b200 as rs
from tests.gpu_util import GpuHandle, dev, host, ptr, ptr_array
from tests.norms import eps_of, norm_error, norm_error_lower, norm_error_upper
from tests.refcases import (from_colmajor, hpd_gram, ref_gesv_input, ref_getrf_input,
                            ref_getrs_input, ref_potrf_input, to_colmajor, uniform_complex)

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "lapack_golden_complex.npz"))
DT = {"z": np.complex128, "c": np.complex64}
OPS = {0: rs.OP_N, 1: rs.OP_T, 2: rs.OP_C}


def eps(P):
    return eps_of(np.float64 if P == "z" else np.float32)


@pytest.fixture(scope="module")
def handle():
    h = GpuHandle()
    yield h.value
    h.close()


def _call(name, *args):
    st = rs.call(name, *args)
    assert st == rs.SUCCESS, (name, rs.STATUS_NAMES[st])


def oracle_getrf(A, pivot=True):
    bc, m, n = A.shape
    mn = max(min(m, n), 1)
    flat = to_colmajor(A)
    ipiv = np.zeros(bc * mn, np.int32)
    info = np.zeros(bc, np.int32)
    oracle.cgetrf(m, n, flat, m, m * n, ipiv, mn, info, bc, pivot)
    return from_colmajor(flat, bc, m, n, m, m * n), ipiv.reshape(bc, -1)[:, :min(m, n)], info


def gpu_getrf(handle, P, A, form="strided", pivot=True, lda=None):
    bc, m, n = A.shape
    lda = m if lda is None else lda
    mn = max(min(m, n), 1)
    dA = dev(to_colmajor(A, lda))
    dP = dev(np.full(bc * mn, -7, np.int32))
    dI = dev(np.full(bc, -7, np.int32))
    npvt = "" if pivot else "_npvt"
    if form == "strided":
        args = [ptr(dA), lda, lda * n] + ([ptr(dP), mn] if pivot else []) + [ptr(dI), bc]
        _call(f"rocsolver_{P}getrf{npvt}_strided_batched", handle, m, n, *args)
    elif form == "batched":
        aA = ptr_array(dA, bc, lda * n)
        args = [ptr(aA), lda] + ([ptr(dP), mn] if pivot else []) + [ptr(dI), bc]
        _call(f"rocsolver_{P}getrf{npvt}_batched", handle, m, n, *args)
    else:
        assert bc == 1
        args = [ptr(dA), lda] + ([ptr(dP)] if pivot else []) + [ptr(dI)]
        _call(f"rocsolver_{P}getrf{npvt}", handle, m, n, *args)
    LU = from_colmajor(host(dA), bc, m, n, lda, lda * n)
    return LU, host(dP).reshape(bc, mn)[:, :min(m, n)], host(dI)


GETRF_CASES = [("z", 32, 16), ("z", 50, 40), ("z", 70, 100), ("c", 50, 40)]


@pytest.mark.parametrize("P,m,n", GETRF_CASES)
@pytest.mark.parametrize("singular", [False, True])
def test_getrf_reference_inputs(handle, P, m, n, singular):
    A = ref_getrf_input(m, n, m, 3, singular, cplx=True).astype(DT[P])
    LU, ipiv, info = gpu_getrf(handle, P, A)
    key = f"{P}getrf_ref_m{m}_n{n}_s{int(singular)}"
    np.testing.assert_array_equal(ipiv, GOLD[key + "_ipiv"])
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    for b in range(3):
        assert norm_error("F", GOLD[key + "_LU"][b], LU[b]) <= min(m, n) * eps(P)


@pytest.mark.parametrize("P", ["c", "z"])
@pytest.mark.parametrize("m,n", [(1, 1), (2, 2), (31, 31), (33, 33), (65, 65), (129, 97),
                                 (97, 129), (300, 300)])
@pytest.mark.parametrize("form", ["strided", "batched"])
def test_getrf_uniform_vs_oracle(handle, P, m, n, form):
    A = uniform_complex(m, n, 3, seed=m * 7 + n).astype(DT[P])
    LU, ipiv, info = gpu_getrf(handle, P, A, form=form, lda=m + 3)
    oLU, oipiv, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(info, oinfo)
    if P == "z" or m <= 65:
        np.testing.assert_array_equal(ipiv, oipiv)
    else:  # FP32 rounding may flip a near tie in |re| + |im|
        assert (ipiv != oipiv).mean() < 0.02
    for b in range(3):
        if np.array_equal(ipiv[b], oipiv[b]):
            assert norm_error("F", oLU[b], LU[b]) <= 4 * min(m, n) * eps(P)


@pytest.mark.parametrize("P", ["c", "z"])
def test_getrf_plain_and_npvt(handle, P):
    A = uniform_complex(40, 40, 1, seed=11).astype(DT[P])
    LU, ipiv, info = gpu_getrf(handle, P, A, form="plain")
    oLU, oipiv, _ = oracle_getrf(A)
    np.testing.assert_array_equal(ipiv, oipiv)
    assert norm_error("F", oLU[0], LU[0]) <= 40 * eps(P)
    # npvt on a diagonally dominant matrix, all three forms
    D = A + 50 * np.eye(40)[None]
    D3 = np.concatenate([D, D * (1 + 1j), D * 2j])
    oLU, _, oinfo = oracle_getrf(D3, pivot=False)
    for form in ("strided", "batched"):
        LU, _, info = gpu_getrf(handle, P, D3.astype(DT[P]), form=form, pivot=False)
        np.testing.assert_array_equal(info, oinfo)
        for b in range(3):
            assert norm_error("F", oLU[b], LU[b]) <= 40 * eps(P)
    LU, _, info = gpu_getrf(handle, P, D.astype(DT[P]), form="plain", pivot=False)
    assert info[0] == 0 and norm_error("F", oLU[0], LU[0]) <= 40 * eps(P)


@pytest.mark.parametrize("P,n,nrhs", [("z", 20, 10), ("z", 50, 30), ("c", 20, 10)])
@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("form", ["strided", "batched", "plain"])
def test_getrs_reference_inputs(handle, P, n, nrhs, trans, form):
    _, B = ref_getrs_input(n, nrhs, 3, cplx=True)
    base = f"{P}getrs_ref_n{n}_r{nrhs}"
    LU = GOLD[base + "_LU"].astype(DT[P])
    ipiv = GOLD[base + "_ipiv"].astype(np.int32)
    X0 = GOLD[f"{base}_t{trans}_X"]
    B = B.astype(DT[P])
    bc = 1 if form == "plain" else 3
    ldb = n + 1
    dA, dB = dev(to_colmajor(LU[:bc])), dev(to_colmajor(B[:bc], ldb))
    dP = dev(ipiv[:bc].reshape(-1).copy())
    if form == "strided":
        _call(f"rocsolver_{P}getrs_strided_batched", handle, OPS[trans], n, nrhs, ptr(dA), n,
              n * n, ptr(dP), n, ptr(dB), ldb, ldb * nrhs, bc)
    elif form == "batched":
        aA, aB = ptr_array(dA, bc, n * n), ptr_array(dB, bc, ldb * nrhs)
        _call(f"rocsolver_{P}getrs_batched", handle, OPS[trans], n, nrhs, ptr(aA), n, ptr(dP),
              n, ptr(aB), ldb, bc)
    else:
        _call(f"rocsolver_{P}getrs", handle, OPS[trans], n, nrhs, ptr(dA), n, ptr(dP), ptr(dB),
              ldb)
    X = from_colmajor(host(dB), bc, n, nrhs, ldb, ldb * nrhs)
    for b in range(bc):
        assert norm_error("I", X0[b], X[b]) <= n * eps(P)


@pytest.mark.parametrize("P", ["c", "z"])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_getrs_uniform_vs_oracle(handle, P, trans):
    n, nrhs = 150, 7
    A = uniform_complex(n, n, 2, seed=77).astype(DT[P])
    B = uniform_complex(n, nrhs, 2, seed=78).astype(DT[P])
    LU, ipiv, _ = oracle_getrf(A)
    fLU = to_colmajor(LU)
    fP = ipiv.reshape(-1).copy()
    oB = to_colmajor(B)
    oracle.cgetrs(trans, n, nrhs, fLU, n, n * n, fP, n, oB, n, n * nrhs, 2)
    dA, dB, dP = dev(fLU), dev(to_colmajor(B)), dev(fP)
    _call(f"rocsolver_{P}getrs_strided_batched", handle, OPS[trans], n, nrhs, ptr(dA), n, n * n,
          ptr(dP), n, ptr(dB), n, n * nrhs, 2)
    X = from_colmajor(host(dB), 2, n, nrhs, n, n * nrhs)
    oX = from_colmajor(oB, 2, n, nrhs, n, n * nrhs)
    for b in range(2):
        # residual check as well: op(A) X = B
        opA = A[b] if trans == 0 else (A[b].T if trans == 1 else np.conj(A[b].T))
        r = np.abs(opA.astype(np.complex128) @ X[b] - B[b]).max()
        assert r <= 1e3 * n * eps(P) * np.abs(X[b]).max()
        assert norm_error("I", oX[b], X[b]) <= 50 * n * eps(P)


@pytest.mark.parametrize("P,n,nrhs", [("z", 20, 1), ("z", 50, 10), ("c", 20, 1)])
@pytest.mark.parametrize("singular", [False, True])
@pytest.mark.parametrize("form", ["strided", "batched"])
def test_gesv_reference_inputs(handle, P, n, nrhs, singular, form):
    A, B = ref_gesv_input(n, nrhs, 3, singular, cplx=True)
    A, B = A.astype(DT[P]), B.astype(DT[P])
    key = f"{P}gesv_ref_n{n}_r{nrhs}_s{int(singular)}"
    dA, dB = dev(to_colmajor(A)), dev(to_colmajor(B))
    dP = dev(np.zeros(3 * n, np.int32))
    dI = dev(np.full(3, -1, np.int32))
    if form == "strided":
        _call(f"rocsolver_{P}gesv_strided_batched", handle, n, nrhs, ptr(dA), n, n * n, ptr(dP),
              n, ptr(dB), n, n * nrhs, ptr(dI), 3)
    else:
        aA, aB = ptr_array(dA, 3, n * n), ptr_array(dB, 3, n * nrhs)
        _call(f"rocsolver_{P}gesv_batched", handle, n, nrhs, ptr(aA), n, ptr(dP), n, ptr(aB), n,
              ptr(dI), 3)
    X = from_colmajor(host(dB), 3, n, nrhs, n, n * nrhs)
    info = host(dI)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    np.testing.assert_array_equal(host(dP).reshape(3, n), GOLD[key + "_ipiv"])
    for b in range(3):
        if info[b] == 0:
            assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * eps(P)
        else:  # B untouched for failed members (roclapack_gesv.hpp:163-176)
            np.testing.assert_array_equal(X[b], B[b])


@pytest.mark.parametrize("P", ["c", "z"])
def test_gesv_plain(handle, P):
    n, nrhs = 45, 3
    A = uniform_complex(n, n, 1, seed=3).astype(DT[P])
    B = uniform_complex(n, nrhs, 1, seed=4).astype(DT[P])
    oA, oB = to_colmajor(A), to_colmajor(B)
    oP, oI = np.zeros(n, np.int32), np.zeros(1, np.int32)
    oracle.cgesv(n, nrhs, oA, n, n * n, oP, n, oB, n, n * nrhs, oI, 1)
    dA, dB = dev(to_colmajor(A)), dev(to_colmajor(B))
    dP, dI = dev(np.zeros(n, np.int32)), dev(np.full(1, -1, np.int32))
    _call(f"rocsolver_{P}gesv", handle, n, nrhs, ptr(dA), n, ptr(dP), ptr(dB), n, ptr(dI))
    assert host(dI)[0] == 0
    np.testing.assert_array_equal(host(dP), oP)
    X = from_colmajor(host(dB), 1, n, nrhs, n, n * nrhs)[0]
    assert norm_error("I", from_colmajor(oB, 1, n, nrhs, n, n * nrhs)[0], X) <= 20 * n * eps(P)


def gpu_potrf(handle, P, A, lower, form="strided", lda=None):
    bc, n, _ = A.shape
    lda = n if lda is None else lda
    dA = dev(to_colmajor(A, lda))
    dI = dev(np.full(bc, -7, np.int32))
    uplo = rs.FILL_LOWER if lower else rs.FILL_UPPER
    if form == "strided":
        _call(f"rocsolver_{P}potrf_strided_batched", handle, uplo, n, ptr(dA), lda, lda * n,
              ptr(dI), bc)
    elif form == "batched":
        aA = ptr_array(dA, bc, lda * n)
        _call(f"rocsolver_{P}potrf_batched", handle, uplo, n, ptr(aA), lda, ptr(dI), bc)
    else:
        _call(f"rocsolver_{P}potrf", handle, uplo, n, ptr(dA), lda, ptr(dI))
    return from_colmajor(host(dA), bc, n, n, lda, lda * n), host(dI), dA


@pytest.mark.parametrize("P,n", [("z", 10), ("z", 50), ("c", 10)])
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("singular", [False, True])
@pytest.mark.parametrize("form", ["strided", "batched"])
def test_potrf_reference_inputs(handle, P, n, lower, singular, form):
    A = ref_potrf_input(n, 3, singular, cplx=True).astype(DT[P])
    C, info, _ = gpu_potrf(handle, P, A, lower, form, lda=n + 2)
    key = f"{P}potrf_ref_n{n}_L{int(lower)}_s{int(singular)}"
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    f = norm_error_lower if lower else norm_error_upper
    for b in range(3):
        nn = n if info[b] == 0 else info[b] - 1
        assert f("F", GOLD[key + "_C"][b][:nn, :nn], C[b][:nn, :nn]) <= n * eps(P)
        # the other triangle is not referenced
        other = np.triu(np.ones((n, n), bool), 1) if lower else np.tril(np.ones((n, n), bool), -1)
        np.testing.assert_array_equal(C[b][other], A[b][other])


@pytest.mark.parametrize("P,n", [("z", 1), ("z", 33), ("z", 64), ("c", 33)])
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("form", ["strided", "batched", "plain"])
def test_potrf_potrs_hermitian(handle, P, n, lower, form):
    A = hpd_gram(n, 4, seed=500 + n).astype(DT[P])
    B = uniform_complex(n, 3, 4, seed=600 + n).astype(DT[P])
    key = f"{P}potrs_hpd_n{n}_L{int(lower)}"
    bc = 1 if form == "plain" else 4
    C, info, dA = gpu_potrf(handle, P, A[:bc], lower, form)
    np.testing.assert_array_equal(info, GOLD[key + "_info"][:bc])
    f = norm_error_lower if lower else norm_error_upper
    for b in range(bc):
        assert f("F", GOLD[key + "_C"][b], C[b]) <= n * eps(P)
    ldb = n + 1
    dB = dev(to_colmajor(B[:bc], ldb))
    uplo = rs.FILL_LOWER if lower else rs.FILL_UPPER
    if form == "strided":
        _call(f"rocsolver_{P}potrs_strided_batched", handle, uplo, n, 3, ptr(dA), n, n * n,
              ptr(dB), ldb, ldb * 3, bc)
    elif form == "batched":
        aA, aB = ptr_array(dA, bc, n * n), ptr_array(dB, bc, ldb * 3)
        _call(f"rocsolver_{P}potrs_batched", handle, uplo, n, 3, ptr(aA), n, ptr(aB), ldb, bc)
    else:
        _call(f"rocsolver_{P}potrs", handle, uplo, n, 3, ptr(dA), n, ptr(dB), ldb)
    X = from_colmajor(host(dB), bc, n, 3, ldb, ldb * 3)
    for b in range(bc):
        assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * eps(P)


@pytest.mark.parametrize("P", ["c", "z"])
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("form", ["strided", "batched", "plain"])
def test_posv(handle, P, lower, form):
    n, nrhs = 40, 2
    bc = 1 if form == "plain" else 3
    A = hpd_gram(n, bc, seed=9).astype(DT[P])
    if bc == 3:  # member 1 not positive definite: info > 0 and its B untouched
        A[1][7, 7] = -1.0
    B = uniform_complex(n, nrhs, bc, seed=10).astype(DT[P])
    oA, oB = to_colmajor(A), to_colmajor(B)
    oI = np.zeros(bc, np.int32)
    oracle.cposv(not lower, n, nrhs, oA, n, n * n, oB, n, n * nrhs, oI, bc)
    dA, dB = dev(to_colmajor(A)), dev(to_colmajor(B))
    dI = dev(np.full(bc, -7, np.int32))
    uplo = rs.FILL_LOWER if lower else rs.FILL_UPPER
    if form == "strided":
        _call(f"rocsolver_{P}posv_strided_batched", handle, uplo, n, nrhs, ptr(dA), n, n * n,
              ptr(dB), n, n * nrhs, ptr(dI), bc)
    elif form == "batched":
        aA, aB = ptr_array(dA, bc, n * n), ptr_array(dB, bc, n * nrhs)
        _call(f"rocsolver_{P}posv_batched", handle, uplo, n, nrhs, ptr(aA), n, ptr(aB), n,
              ptr(dI), bc)
    else:
        _call(f"rocsolver_{P}posv", handle, uplo, n, nrhs, ptr(dA), n, ptr(dB), n, ptr(dI))
    info = host(dI)
    np.testing.assert_array_equal(info, oI)
    X = from_colmajor(host(dB), bc, n, nrhs, n, n * nrhs)
    oX = from_colmajor(oB, bc, n, nrhs, n, n * nrhs)
    for b in range(bc):
        if info[b] == 0:
            assert norm_error("I", oX[b], X[b]) <= 10 * n * eps(P)
        else:
            np.testing.assert_array_equal(X[b], B[b])


@pytest.mark.parametrize("P", ["c", "z"])
def test_nan_and_zero_pivots(handle, P):
    """A NaN in the first candidate row wins the pivot search, one elsewhere never does
    (LAPACK izamax); an exactly zero column sets info to its order and the factorisation
    goes on."""
    n = 24
    A = uniform_complex(n, n, 3, seed=21).astype(DT[P])
    A[0][0, 0] = complex(np.nan, 0)
    A[1][5, 0] = complex(0, np.nan)
    A[2][:, 9] = 0
    LU, ipiv, info = gpu_getrf(handle, P, A)
    oLU, oipiv, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(ipiv[:, :1], oipiv[:, :1])
    np.testing.assert_array_equal(info, oinfo)
    assert info[2] == 10
    np.testing.assert_array_equal(ipiv[2], oipiv[2])
    assert norm_error("F", oLU[2], LU[2]) <= n * eps(P)


@pytest.mark.parametrize("P", ["c", "z"])
def test_empty_and_quick_returns(handle, P):
    dI = dev(np.full(2, -7, np.int32))
    dA = dev(np.zeros(4, DT[P]))
    _call(f"rocsolver_{P}getrf_strided_batched", handle, 0, 3, ptr(dA), 1, 0, ptr(dI), 1,
          ptr(dI), 2)
    np.testing.assert_array_equal(host(dI), [0, 0])
    dI = dev(np.full(2, -7, np.int32))
    _call(f"rocsolver_{P}potrf_strided_batched", handle, rs.FILL_LOWER, 0, ptr(dA), 1, 0, ptr(dI),
          2)
    np.testing.assert_array_equal(host(dI), [0, 0])
    _call(f"rocsolver_{P}getrs_strided_batched", handle, rs.OP_C, 0, 1, None, 1, 0, None, 1,
          None, 1, 0, 2)


@pytest.mark.parametrize("P", ["c", "z"])
@pytest.mark.parametrize("n", [70, 257, 300])
def test_kernel_boundaries(handle, P, n):
    """Sizes on both sides of the shared-memory factorisation limit (96 KB per member) and of
    the warp solves (n <= 256): getrf, getrs with N / T / C and potrf / potrs (lower and
    upper) against the oracle."""
    bc, nrhs = 2, 3
    A = uniform_complex(n, n, bc, seed=900 + n).astype(DT[P])
    B = uniform_complex(n, nrhs, bc, seed=901 + n).astype(DT[P])
    LU, ipiv, info = gpu_getrf(handle, P, A)
    oLU, oipiv, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(info, oinfo)
    if P == "z":
        np.testing.assert_array_equal(ipiv, oipiv)
    for b in range(bc):
        if np.array_equal(ipiv[b], oipiv[b]):
            assert norm_error("F", oLU[b], LU[b]) <= 4 * n * eps(P)
    fLU, fP = to_colmajor(LU), ipiv.reshape(-1).astype(np.int32).copy()
    for trans in (0, 1, 2):
        oB = to_colmajor(B)
        oracle.cgetrs(trans, n, nrhs, fLU.copy(), n, n * n, fP.copy(), n, oB, n, n * nrhs, bc)
        dA, dB, dP = dev(fLU), dev(to_colmajor(B)), dev(fP)
        _call(f"rocsolver_{P}getrs_strided_batched", handle, OPS[trans], n, nrhs, ptr(dA), n,
              n * n, ptr(dP), n, ptr(dB), n, n * nrhs, bc)
        X = from_colmajor(host(dB), bc, n, nrhs, n, n * nrhs)
        oX = from_colmajor(oB, bc, n, nrhs, n, n * nrhs)
        for b in range(bc):
            assert norm_error("I", oX[b], X[b]) <= 20 * n * eps(P), (trans, b)
    H = hpd_gram(n, bc, seed=902 + n).astype(DT[P])
    for lower in (True, False):
        C, info, dC = gpu_potrf(handle, P, H, lower)
        oC = to_colmajor(H)
        oI = np.zeros(bc, np.int32)
        oracle.cpotrf(not lower, n, oC, n, n * n, oI, bc)
        np.testing.assert_array_equal(info, oI)
        f = norm_error_lower if lower else norm_error_upper
        oCm = from_colmajor(oC, bc, n, n, n, n * n)
        for b in range(bc):
            assert f("F", oCm[b], C[b]) <= n * eps(P)
        dB = dev(to_colmajor(B))
        uplo = rs.FILL_LOWER if lower else rs.FILL_UPPER
        _call(f"rocsolver_{P}potrs_strided_batched", handle, uplo, n, nrhs, ptr(dC), n, n * n,
              ptr(dB), n, n * nrhs, bc)
        oB = to_colmajor(B)
        oracle.cpotrs(not lower, n, nrhs, oC, n, n * n, oB, n, n * nrhs, bc)
        X = from_colmajor(host(dB), bc, n, nrhs, n, n * nrhs)
        oX = from_colmajor(oB, bc, n, nrhs, n, n * nrhs)
        for b in range(bc):
            assert norm_error("I", oX[b], X[b]) <= 20 * n * eps(P), (lower, b)


@pytest.mark.parametrize("P", ["c", "z"])
@pytest.mark.parametrize("m,n", [(20, 7), (7, 20), (32, 32), (9, 16), (17, 5)])
@pytest.mark.parametrize("pivot", [True, False])
def test_warp_lu_small_shapes(handle, P, m, n, pivot):
    """The one-warp-per-member LU (m, n <= 32): rectangular shapes, padded leading dimension,
    with and without pivoting, against the oracle."""
    A = uniform_complex(m, n, 5, seed=m * 31 + n).astype(DT[P])
    if not pivot:
        for b in range(5):
            A[b][np.arange(min(m, n)), np.arange(min(m, n))] += 8.0
    LU, ipiv, info = gpu_getrf(handle, P, A, pivot=pivot, lda=m + 2)
    oLU, oipiv, oinfo = oracle_getrf(A, pivot=pivot)
    np.testing.assert_array_equal(info, oinfo)
    if pivot:
        np.testing.assert_array_equal(ipiv, oipiv)
    for b in range(5):
        assert norm_error("F", oLU[b], LU[b]) <= 4 * max(m, n) * eps(P)


@pytest.mark.parametrize("P", ["c", "z"])
@pytest.mark.parametrize("m,n", [(33, 33), (64, 64), (64, 33), (33, 64), (20, 64), (64, 20),
                                 (40, 63), (57, 48)])
@pytest.mark.parametrize("pivot", [True, False])
def test_register_lu_shapes(handle, P, m, n, pivot):
    """The register-resident LU (m, n <= 64, not both <= 32; one CTA per member, warps over
    column groups): rectangular shapes either way, one or two rows per lane, padded leading
    dimension, with and without pivoting, against the oracle."""
    A = uniform_complex(m, n, 6, seed=m * 67 + n).astype(DT[P])
    if not pivot:
        for b in range(6):
            A[b][np.arange(min(m, n)), np.arange(min(m, n))] += 8.0
    LU, ipiv, info = gpu_getrf(handle, P, A, pivot=pivot, lda=m + 3)
    oLU, oipiv, oinfo = oracle_getrf(A, pivot=pivot)
    np.testing.assert_array_equal(info, oinfo)
    if pivot:
        np.testing.assert_array_equal(ipiv, oipiv)
    for b in range(6):
        assert norm_error("F", oLU[b], LU[b]) <= 4 * max(m, n) * eps(P)


@pytest.mark.parametrize("P", ["c", "z"])
def test_register_lu_nan_zero_and_ties(handle, P):
    """n = 48 (register LU): a NaN in the first candidate row wins, one elsewhere never does;
    a zero column sets info and the factorisation goes on; equal magnitudes pick the first
    row in position order (LAPACK izamax) after earlier interchanges."""
    n = 48
    A = uniform_complex(n, n, 4, seed=77).astype(DT[P])
    A[0][0, 0] = complex(np.nan, 0)
    A[1][40, 0] = complex(0, np.nan)
    A[2][:, 35] = 0
    A[3][:, :] = np.round(A[3] * 2) / 2  # many exact ties in |re| + |im|
    LU, ipiv, info = gpu_getrf(handle, P, A)
    oLU, oipiv, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(ipiv[:, :1], oipiv[:, :1])
    np.testing.assert_array_equal(info, oinfo)
    assert info[2] == 36
    for b in (2, 3):
        np.testing.assert_array_equal(ipiv[b], oipiv[b])
        assert norm_error("F", oLU[b], LU[b]) <= n * eps(P)


@pytest.mark.parametrize("P", ["c", "z"])
@pytest.mark.parametrize("n", [1, 5, 17, 32])
@pytest.mark.parametrize("lower", [True, False])
def test_warp_cholesky_small(handle, P, n, lower):
    """Small Hermitian Cholesky (n <= 32, padded leading dimension): factors against the
    oracle in the referenced triangle, the other triangle untouched, and a member that is not
    positive definite (info, the failing pivot stored, later columns untouched)."""
    bc = 4
    A = hpd_gram(n, bc, seed=700 + n).astype(DT[P])
    if n > 2:
        A[2][n // 2, n // 2] = -1.0
    C, info, _ = gpu_potrf(handle, P, A, lower, lda=n + 3)
    oC = to_colmajor(A)
    oI = np.zeros(bc, np.int32)
    oracle.cpotrf(not lower, n, oC, n, n * n, oI, bc)
    oCm = from_colmajor(oC, bc, n, n, n, n * n)
    np.testing.assert_array_equal(info, oI)
    f = norm_error_lower if lower else norm_error_upper
    other = np.triu(np.ones((n, n), bool), 1) if lower else np.tril(np.ones((n, n), bool), -1)
    for b in range(bc):
        nn = n if info[b] == 0 else info[b] - 1
        assert f("F", oCm[b][:nn, :nn], C[b][:nn, :nn]) <= n * eps(P)
        np.testing.assert_array_equal(C[b][other], A[b][other])
        if info[b] != 0:  # the failing pivot is stored; the columns after it keep A
            k = info[b] - 1
            assert abs(C[b][k, k] - oCm[b][k, k]) <= 1e3 * eps(P) * abs(oCm[b][k, k])
            tail = np.tril(np.ones((n, n), bool), -1) if lower else np.triu(np.ones((n, n), bool), 1)
            cols = np.zeros((n, n), bool)
            if lower:
                cols[:, k:] = True
            else:
                cols[k:, :] = True
            np.testing.assert_array_equal(C[b][tail & cols], A[b][tail & cols])


# ---------------------------------------------------------------- getri and gesv_outofplace
@pytest.mark.parametrize("key", [c for c in [str(x) for x in GOLD["cases"]]
                                 if c[1:].startswith("getri")])
@pytest.mark.parametrize("form", ["strided", "batched", "outofplace"])
def test_getri_reference_inputs(handle, key, form):
    """c / z getri from the golden LAPACK factors: info exact, inverse within n*eps (F-norm);
    singular members keep their factors (getri_outofplace: C = I, as the real path)."""
    P = key[0]
    n = int(key.split("_n")[1].split("_")[0])
    LU = GOLD[key + "_LU"].astype(DT[P])
    ipiv = GOLD[key + "_ipiv"].astype(np.int32).reshape(-1).copy()
    dA = dev(to_colmajor(LU, n + 1))
    dP = dev(ipiv)
    dI = dev(np.full(3, -7, np.int32))
    lda = n + 1
    if form == "strided":
        _call(f"rocsolver_{P}getri_strided_batched", handle, n, ptr(dA), lda, lda * n, ptr(dP), n,
              ptr(dI), 3)
        out = from_colmajor(host(dA), 3, n, n, lda, lda * n)
    elif form == "batched":
        aA = ptr_array(dA, 3, lda * n)
        _call(f"rocsolver_{P}getri_batched", handle, n, ptr(aA), lda, ptr(dP), n, ptr(dI), 3)
        out = from_colmajor(host(dA), 3, n, n, lda, lda * n)
    else:
        dC = dev(np.zeros(3 * n * n, DT[P]))
        _call(f"rocsolver_{P}getri_outofplace_strided_batched", handle, n, ptr(dA), lda, lda * n,
              ptr(dP), n, ptr(dC), n, n * n, ptr(dI), 3)
        out = from_colmajor(host(dC), 3, n, n, n, n * n)
    info = host(dI)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    for b in range(3):
        if info[b] == 0:
            assert norm_error("F", GOLD[key + "_inv"][b], out[b]) <= 4 * n * eps(P)
        elif form == "outofplace":
            np.testing.assert_array_equal(out[b], np.eye(n))
        else:
            np.testing.assert_array_equal(out[b], LU[b])


@pytest.mark.parametrize("P", ["c", "z"])
@pytest.mark.parametrize("n", [1, 7, 32, 33, 100, 256, 300])
@pytest.mark.parametrize("pivot", [True, False])
def test_getri_vs_oracle(handle, P, n, pivot):
    """c / z getri (in place, with and without pivoting) against the complex oracle."""
    A = (uniform_complex(n, n, 2, seed=4200 + n) + 2 * n * np.eye(n)[None]).astype(DT[P])
    LU, ipiv, info = gpu_getrf(handle, P, A, pivot=pivot)
    assert not info.any()
    f = to_colmajor(LU)
    fP = ipiv.reshape(-1).astype(np.int32).copy()
    oI = np.zeros(2, np.int32)
    oracle.cgetri(n, f, n, n * n, fP, n, oI, 2, pivot=pivot)
    ref = from_colmajor(f, 2, n, n, n, n * n)
    dA, dI, dP = dev(to_colmajor(LU)), dev(np.full(2, -7, np.int32)), dev(fP)
    if pivot:
        _call(f"rocsolver_{P}getri_strided_batched", handle, n, ptr(dA), n, n * n, ptr(dP), n,
              ptr(dI), 2)
    else:
        _call(f"rocsolver_{P}getri_npvt_strided_batched", handle, n, ptr(dA), n, n * n, ptr(dI),
              2)
    np.testing.assert_array_equal(host(dI), oI)
    inv = from_colmajor(host(dA), 2, n, n, n, n * n)
    for b in range(2):
        assert norm_error("F", ref[b], inv[b]) <= 8 * n * eps(P)


@pytest.mark.parametrize("P", ["c", "z"])
@pytest.mark.parametrize("n", [5, 32, 64])
def test_gesv_outofplace(handle, P, n):
    """X = A^{-1} B with B left as it was; A and ipiv hold the factors (zgesv's)."""
    nrhs = 3
    A = uniform_complex(n, n, 1, seed=77 + n).astype(DT[P])
    B = uniform_complex(n, nrhs, 1, seed=78 + n).astype(DT[P])
    oA, oB = to_colmajor(A), to_colmajor(B)
    oP, oI = np.zeros(n, np.int32), np.zeros(1, np.int32)
    oracle.cgesv(n, nrhs, oA, n, n * n, oP, n, oB, n, n * nrhs, oI, 1)
    dA, dB, dX = dev(to_colmajor(A)), dev(to_colmajor(B)), dev(np.zeros(n * nrhs, DT[P]))
    dP, dI = dev(np.zeros(n, np.int32)), dev(np.full(1, -7, np.int32))
    _call(f"rocsolver_{P}gesv_outofplace", handle, n, nrhs, ptr(dA), n, ptr(dP), ptr(dB), n,
          ptr(dX), n, ptr(dI))
    assert host(dI)[0] == 0
    np.testing.assert_array_equal(host(dP), oP)
    np.testing.assert_array_equal(host(dB), to_colmajor(B))
    X = from_colmajor(host(dX), 1, n, nrhs, n, n * nrhs)[0]
    assert norm_error("I", from_colmajor(oB, 1, n, nrhs, n, n * nrhs)[0], X) <= 20 * n * eps(P)
