"""Pin the complex oracle (oracle/oracle_complex.c): on the committed golden fixtures made by
host LAPACK (zgetrf, zgetrs, zpotrf, zpotrs, zgesv and the c routines; the reference's clients
compare against the same routines, clients/common/lapack_host_reference.cpp), with the
reference's acceptance rules: ipiv and info exact, factors within min(m,n)*eps (F-norm) and
solutions within n*eps (inf-norm) (clients/include/testing_getf2_getrf.hpp:233-259,
testing_getrs.hpp:219-229, testing_potf2_potrf.hpp:186-210, testing_gesv.hpp:229-247).
Complex inputs of the reference's suites take two draws of its integer stream per element."""
import os

import numpy as np
import pytest

import oracle
from tests.norms import eps_of, norm_error, norm_error_lower, norm_error_upper
from tests.refcases import (from_colmajor, hpd_gram, ref_gesv_input, ref_getrf_input,
                            ref_getrs_input, ref_potrf_input, to_colmajor, uniform_complex)

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "lapack_golden_complex.npz"))
CASES = [str(c) for c in GOLD["cases"]]
DT = {"z": np.complex128, "c": np.complex64}


def _parse(key):
    parts = key.split("_")
    kv = {}
    for p in parts[2:]:
        k = p.rstrip("0123456789")
        kv[k] = int(p[len(k):])
    return parts[0][0], parts[0][1:], parts[1], kv


def _eps(P):
    return eps_of(np.float64 if P == "z" else np.float32)


def cplx_getrf(A, pivot=True):
    bc, m, n = A.shape
    mn = max(min(m, n), 1)
    flat = to_colmajor(A)
    ipiv = np.zeros(bc * mn, np.int32)
    info = np.zeros(bc, np.int32)
    oracle.cgetrf(m, n, flat, m, m * n, ipiv, mn, info, bc, pivot)
    return from_colmajor(flat, bc, m, n, m, m * n), ipiv.reshape(bc, -1)[:, :min(m, n)], info


@pytest.mark.parametrize("key", [c for c in CASES if c[1:].startswith("getrf")])
def test_complex_oracle_getrf_matches_lapack(key):
    P, _, kind, kv = _parse(key)
    if kind == "ref":
        m, n = kv["m"], kv["n"]
        A = ref_getrf_input(m, n, m, 3, bool(kv["s"]), cplx=True)
    else:
        m = n = kv["n"]
        A = uniform_complex(n, n, 4, seed=400 + n)
    A = A.astype(DT[P])
    LU, ipiv, info = cplx_getrf(A)
    np.testing.assert_array_equal(ipiv, GOLD[key + "_ipiv"])
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    for b in range(A.shape[0]):
        assert norm_error("F", GOLD[key + "_LU"][b], LU[b]) <= min(m, n) * _eps(P)


@pytest.mark.parametrize("key", [c for c in CASES if c[1:].startswith("getrs")])
def test_complex_oracle_getrs_matches_lapack(key):
    P, _, _, kv = _parse(key)
    n, nrhs, trans = kv["n"], kv["r"], kv["t"]
    _, B = ref_getrs_input(n, nrhs, 3, cplx=True)
    base = f"{P}getrs_ref_n{n}_r{nrhs}"
    LU = to_colmajor(GOLD[base + "_LU"])
    ipiv = GOLD[base + "_ipiv"].astype(np.int32).reshape(-1).copy()
    Bf = to_colmajor(B.astype(DT[P]))
    oracle.cgetrs(trans, n, nrhs, LU, n, n * n, ipiv, n, Bf, n, n * nrhs, 3)
    X = from_colmajor(Bf, 3, n, nrhs, n, n * nrhs)
    for b in range(3):
        assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * _eps(P)


@pytest.mark.parametrize("key", [c for c in CASES if c[1:].startswith(("potrf", "potrs"))])
def test_complex_oracle_potrf_potrs_matches_lapack(key):
    P, op, kind, kv = _parse(key)
    n, lower = kv["n"], bool(kv["L"])
    if kind == "ref":
        A = ref_potrf_input(n, 3, bool(kv["s"]), cplx=True)
    else:
        A = hpd_gram(n, 4, seed=500 + n)
    A = A.astype(DT[P])
    bc = A.shape[0]
    flat = to_colmajor(A)
    info = np.zeros(bc, np.int32)
    oracle.cpotrf(not lower, n, flat, n, n * n, info, bc)
    C = from_colmajor(flat, bc, n, n, n, n * n)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    f = norm_error_lower if lower else norm_error_upper
    for b in range(bc):
        nn = n if info[b] == 0 else info[b] - 1  # columns factored before the failure
        assert f("F", GOLD[key + "_C"][b][:nn, :nn], C[b][:nn, :nn]) <= n * _eps(P)
    if op == "potrs":
        B = uniform_complex(n, 3, 4, seed=600 + n).astype(DT[P])
        Bf = to_colmajor(B)
        oracle.cpotrs(not lower, n, 3, flat, n, n * n, Bf, n, n * 3, bc)
        X = from_colmajor(Bf, bc, n, 3, n, n * 3)
        for b in range(bc):
            assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * _eps(P)


@pytest.mark.parametrize("key", [c for c in CASES if c[1:].startswith("gesv")])
def test_complex_oracle_gesv_matches_lapack(key):
    P, _, _, kv = _parse(key)
    n, nrhs, singular = kv["n"], kv["r"], bool(kv["s"])
    A, B = ref_gesv_input(n, nrhs, 3, singular, cplx=True)
    A, B = A.astype(DT[P]), B.astype(DT[P])
    Af, Bf = to_colmajor(A), to_colmajor(B)
    ipiv = np.zeros(3 * n, np.int32)
    info = np.zeros(3, np.int32)
    oracle.cgesv(n, nrhs, Af, n, n * n, ipiv, n, Bf, n, n * nrhs, info, 3)
    X = from_colmajor(Bf, 3, n, nrhs, n, n * nrhs)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    np.testing.assert_array_equal(ipiv.reshape(3, n), GOLD[key + "_ipiv"])
    for b in range(3):
        if info[b] == 0:
            assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * _eps(P)
        else:  # B untouched for failed members (roclapack_gesv.hpp:163-176)
            np.testing.assert_array_equal(X[b], B[b])


def test_complex_reference_stream_pairs():
    """Complex suite inputs: real part from the even draws, imaginary from the odd ones."""
    from tests.refcases import _refstream
    v = oracle.refgen(20)
    z = _refstream(10, cplx=True)
    np.testing.assert_array_equal(z.real, v[0::2])
    np.testing.assert_array_equal(z.imag, v[1::2])


@pytest.mark.parametrize("key", [c for c in CASES if c[1:].startswith("getri")])
def test_complex_oracle_getri_matches_lapack(key):
    """zgetri / cgetri from the golden factors: info exact, inverse within n*eps (F-norm,
    relative); singular members keep their factors."""
    P, _, _, kv = _parse(key)
    n = kv["n"]
    LU = GOLD[key + "_LU"]
    f = to_colmajor(LU)
    ipiv = GOLD[key + "_ipiv"].astype(np.int32).reshape(-1).copy()
    info = np.zeros(3, np.int32)
    oracle.cgetri(n, f, n, n * n, ipiv, n, info, 3)
    inv = from_colmajor(f, 3, n, n, n, n * n)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    for b in range(3):
        if info[b] == 0:
            assert norm_error("F", GOLD[key + "_inv"][b], inv[b]) <= n * _eps(P)
        else:
            np.testing.assert_array_equal(inv[b], LU[b])
