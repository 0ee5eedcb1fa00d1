"""Pin the oracle: the CPU restatement must reproduce host LAPACK (the
reference's own test oracle) on the committed golden fixtures, with the
reference's acceptance rules: ipiv and info exact, factors within
min(m,n)*eps (F-norm) and solutions within n*eps (inf-norm)
(clients/include/testing_getf2_getrf.hpp:233-259,504; testing_getrs.hpp:219-229,462;
testing_potf2_potrf.hpp:186-210,450; testing_gesv.hpp:229-247,506)."""
import os

import numpy as np
import pytest

import oracle
from tests.norms import eps_of, norm_error, norm_error_lower, norm_error_upper
from tests.refcases import (cond_graded, from_colmajor, projections, ref_gesv_input,
                            ref_getrf_input, ref_getrs_input, ref_potrf_input, spd_gram,
                            to_colmajor, uniform_general)

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "lapack_golden.npz"))
CASES = [str(c) for c in GOLD["cases"]]
EPS = eps_of(np.float64)


def _parse(key):
    parts = key.split("_")
    kv = {}
    for p in parts[2:]:
        k = p.rstrip("0123456789")
        kv[k] = int(p[len(k):])
    return parts[0], parts[1], kv


def _oracle_getrf(A):
    bc, m, n = A.shape
    flat = to_colmajor(A)
    ipiv = np.zeros(bc * max(min(m, n), 1), np.int32)
    info = np.zeros(bc, np.int32)
    oracle.getrf(m, n, flat, m, m * n, ipiv, max(min(m, n), 1), info, bc)
    return from_colmajor(flat, bc, m, n, m, m * n), ipiv.reshape(bc, -1)[:, :min(m, n)], info


@pytest.mark.parametrize("key", [c for c in CASES if c.startswith("getrf")])
def test_oracle_getrf_matches_lapack(key):
    _, kind, kv = _parse(key)
    if kind == "ref":
        m, n = kv["m"], kv["n"]
        A = ref_getrf_input(m, n, m, 3, bool(kv["s"]))
    else:
        m = n = kv["n"]
        A = uniform_general(n, n, 4, seed=100 + n)
    LU, ipiv, info = _oracle_getrf(A)
    np.testing.assert_array_equal(ipiv, GOLD[key + "_ipiv"])
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    for b in range(A.shape[0]):
        assert norm_error("F", GOLD[key + "_LU"][b], LU[b]) <= min(m, n) * EPS


@pytest.mark.parametrize("key", [c for c in CASES if c.startswith("getrs")])
def test_oracle_getrs_matches_lapack(key):
    _, _, kv = _parse(key)
    n, nrhs, trans = kv["n"], kv["r"], kv["t"]
    _, B = ref_getrs_input(n, nrhs, 3)
    LU = to_colmajor(GOLD[key + "_LU"])
    ipiv = GOLD[key + "_ipiv"].astype(np.int32).reshape(-1).copy()
    Bf = to_colmajor(B)
    oracle.getrs(trans, n, nrhs, LU, n, n * n, ipiv, n, Bf, n, n * nrhs, 3)
    X = from_colmajor(Bf, 3, n, nrhs, n, n * nrhs)
    for b in range(3):
        assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * EPS


@pytest.mark.parametrize("key", [c for c in CASES if c.startswith("potrf") or c.startswith("potrs")])
def test_oracle_potrf_potrs_matches_lapack(key):
    op, kind, kv = _parse(key)
    n, lower = kv["n"], bool(kv["L"])
    if kind == "ref":
        A = ref_potrf_input(n, 3, bool(kv["s"]))
    else:
        A = spd_gram(n, 4, seed=200 + n)
    bc = A.shape[0]
    flat = to_colmajor(A)
    info = np.zeros(bc, np.int32)
    oracle.potrf(not lower, n, flat, n, n * n, info, bc)
    C = from_colmajor(flat, bc, n, n, n, n * n)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    for b in range(bc):
        nn = n if info[b] == 0 else info[b]
        f = norm_error_lower if lower else norm_error_upper
        assert f("F", GOLD[key + "_C"][b][:nn, :nn], C[b][:nn, :nn]) <= n * EPS
    if op == "potrs":
        B = np.random.default_rng(300 + n).standard_normal((4, n, 4))
        Bf = to_colmajor(B)
        oracle.potrs(not lower, n, 4, flat, n, n * n, Bf, n, n * 4, bc)
        X = from_colmajor(Bf, bc, n, 4, n, n * 4)
        for b in range(bc):
            assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * EPS


@pytest.mark.parametrize("key", [c for c in CASES if c.startswith("gesv")])
def test_oracle_gesv_matches_lapack(key):
    _, _, kv = _parse(key)
    n, nrhs, singular = kv["n"], kv["r"], bool(kv["s"])
    A, B = ref_gesv_input(n, nrhs, 3, singular)
    Af, Bf = to_colmajor(A), to_colmajor(B)
    ipiv = np.zeros(3 * n, np.int32)
    info = np.zeros(3, np.int32)
    oracle.gesv(n, nrhs, Af, n, n * n, ipiv, n, Bf, n, n * nrhs, info, 3)
    X = from_colmajor(Bf, 3, n, nrhs, n, n * nrhs)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    np.testing.assert_array_equal(ipiv.reshape(3, n), GOLD[key + "_ipiv"])
    for b in range(3):
        if info[b] == 0:
            assert norm_error("I", GOLD[key + "_X"][b], X[b]) <= n * EPS
        else:  # B untouched for failed members (roclapack_gesv.hpp:163-176)
            np.testing.assert_array_equal(X[b], B[b])


def test_refgen_is_reference_stream():
    """mt19937(69069) + uniform_int_distribution<int>(1,10): values are integers in
    [1,10], the stream restarts on every reset, and it is roughly uniform."""
    v = oracle.refgen(20000)
    assert np.all(v == np.round(v)) and v.min() == 1 and v.max() == 10
    np.testing.assert_array_equal(v[:100], oracle.refgen(100))
    counts = np.bincount(v.astype(int))[1:]
    assert counts.min() > 1800 and counts.max() < 2200


def test_oracle_batch_threads_agree():
    A = uniform_general(40, 40, 16, seed=7)
    f1, f2 = to_colmajor(A), to_colmajor(A)
    p1, p2 = np.zeros(16 * 40, np.int32), np.zeros(16 * 40, np.int32)
    i1, i2 = np.zeros(16, np.int32), np.zeros(16, np.int32)
    oracle.getrf(40, 40, f1, 40, 1600, p1, 40, i1, 16, nthreads=1)
    oracle.getrf(40, 40, f2, 40, 1600, p2, 40, i2, 16, nthreads=4)
    np.testing.assert_array_equal(f1, f2)
    np.testing.assert_array_equal(p1, p2)


# ---- large members at the benchmarked orders (n = 256, 512; the mixed-precision
# configuration's cond-graded inputs): ipiv and info exact, the factors through their
# projections LU V and W^T LU (the fixture keeps those, not the factors)
def _big_input(key):
    _, kind, kv = _parse(key)
    n = kv["n"]
    if kind == "cond":
        return cond_graded(n, 3, seed=2000 + n)
    return uniform_general(n, n, 2 if n == 256 else 1, seed=1000 + n)


@pytest.mark.parametrize("key", [c for c in CASES if c.startswith("bigrf")])
def test_oracle_large_getrf_matches_lapack(key):
    A = _big_input(key)
    n = A.shape[1]
    LU, ipiv, info = _oracle_getrf(A)
    np.testing.assert_array_equal(ipiv, GOLD[key + "_ipiv"])
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    for b in range(A.shape[0]):
        p, q, V, W = projections(LU[b])
        nrm = np.linalg.norm(LU[b])
        # ||LU_oracle - LU_lapack||_F <= n eps ||LU|| bounds each projection's error by
        # n eps ||LU||_F ||V||_F
        assert np.linalg.norm(p - GOLD[key + "_P"][b]) <= n * EPS * nrm * np.linalg.norm(V)
        assert np.linalg.norm(q - GOLD[key + "_Q"][b]) <= n * EPS * nrm * np.linalg.norm(W)


def test_oracle_large_getrs_matches_lapack():
    A = uniform_general(256, 256, 2, seed=1256)
    B = np.random.default_rng(1257).uniform(-1, 1, (2, 256, 4))
    Af, Bf = to_colmajor(A), to_colmajor(B)
    ipiv = np.zeros(2 * 256, np.int32)
    info = np.zeros(2, np.int32)
    oracle.gesv(256, 4, Af, 256, 256 * 256, ipiv, 256, Bf, 256, 256 * 4, info, 2)
    X = from_colmajor(Bf, 2, 256, 4, 256, 256 * 4)
    np.testing.assert_array_equal(ipiv.reshape(2, 256), GOLD["bigrf_uni_n256_ipiv"])
    for b in range(2):
        # the reference's n eps bound on the solution assumes its diagonally dominant inputs;
        # for uniform members the two solutions differ by up to cond(A) times the backward
        # error, so the test bounds the backward error by n eps and the difference by
        # n eps cond(A)
        kappa = np.linalg.cond(A[b], np.inf)
        res = np.abs(A[b] @ X[b] - B[b]).max()
        assert res <= 256 * EPS * np.abs(A[b]).sum(1).max() * np.abs(X[b]).max()
        assert norm_error("I", GOLD["bigrs_uni_n256_r4_X"][b], X[b]) <= 256 * EPS * kappa


@pytest.mark.parametrize("key", [c for c in CASES if c.startswith("getri")])
def test_oracle_getri_matches_lapack(key):
    """Inverse from the reference's getri inputs: info exact, inverse within n*eps (F-norm,
    clients/include/testing_getri.hpp:209-233)."""
    _, _, kv = _parse(key)
    n = kv["n"]
    LU = GOLD[key + "_LU"]
    flat = to_colmajor(LU)
    ipiv = GOLD[key + "_ipiv"].astype(np.int32).reshape(-1).copy()
    info = np.zeros(3, np.int32)
    oracle.getri(n, flat, n, n * n, ipiv, n, info, 3)
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    inv = from_colmajor(flat, 3, n, n, n, n * n)
    for b in range(3):
        if info[b] == 0:
            assert norm_error("F", GOLD[key + "_inv"][b], inv[b]) <= n * EPS
        else:  # LAPACK leaves the factors in place
            np.testing.assert_array_equal(inv[b], LU[b])
