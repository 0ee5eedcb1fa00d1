"""GPU parity at the benchmarked configurations' own inputs and sizes, and the entry points
no other test file calls.

* dgetrf at n = 256 and 512 against the golden LAPACK fixtures (ipiv and info exact, the
  factors through their projections), and against the oracle on the first 256 members of
  the mixed-precision configuration's own cond-graded inputs (generated exactly as the
  benchmark generates them);
* rocsolver_dgesv_vbatched at the variable-size configuration's shape (n ~ U[8, 512],
  nrhs ~ U[1, 16], A ~ U[-1, 1] + 0.1 n I, max_n 512) against the oracle member by member;
* the non-batched forms rocsolver_{s,d}{getrf,getrs,gesv,potrf,potrs,posv} and
  rocsolver_{s,d}posv_batched.

Acceptance rules are the reference's (clients/include/testing_getf2_getrf.hpp:233-259:
ipiv and info exact; testing_gesv.hpp:229-247 and testing_posv.hpp: B unchanged for
failed members) plus backward errors below 10 n eps."""
import os

import numpy as np
import pytest

import oracle
import rocsolver_b200 as rs
from tests.gpu_util import GpuHandle, dev, host, prefix, ptr, ptr_array
from tests.norms import eps_of, lu_backward_error, solve_backward_error
from tests.refcases import (cond_graded, from_colmajor, projections, spd_gram, to_colmajor,
                            uniform_general)

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "lapack_golden.npz"))
NT = oracle.nthreads_default()


@pytest.fixture(scope="module")
def handle():
    h = GpuHandle()
    yield h.value
    h.close()


def _getrf(handle, A):
    bc, n, _ = A.shape
    dA = dev(to_colmajor(A))
    dP = dev(np.full(bc * n, -7, np.int32))
    dI = dev(np.full(bc, -7, np.int32))
    p = prefix(A.dtype)
    st = rs.call(f"rocsolver_{p}getrf_strided_batched", handle, n, n, ptr(dA), n, n * n,
                 ptr(dP), n, ptr(dI), bc)
    assert st == rs.SUCCESS, rs.STATUS_NAMES[st]
    return from_colmajor(host(dA), bc, n, n, n, n * n), host(dP).reshape(bc, n), host(dI)


# ------------------------------------------------------------------ large golden members
@pytest.mark.parametrize("key", ["bigrf_uni_n256", "bigrf_uni_n512", "bigrf_cond_n256"])
def test_getrf_large_golden(handle, key):
    n = int(key.rsplit("_n", 1)[1])
    A = (cond_graded(n, 3, seed=2000 + n) if "cond" in key
         else uniform_general(n, n, 2 if n == 256 else 1, seed=1000 + n))
    LU, ipiv, info = _getrf(handle, A)
    np.testing.assert_array_equal(ipiv, GOLD[key + "_ipiv"])
    np.testing.assert_array_equal(info, GOLD[key + "_info"])
    eps = eps_of(np.float64)
    for b in range(A.shape[0]):
        p, q, V, W = projections(LU[b])
        nrm = np.linalg.norm(LU[b])
        assert np.linalg.norm(p - GOLD[key + "_P"][b]) <= 4 * n * eps * nrm * np.linalg.norm(V)
        assert np.linalg.norm(q - GOLD[key + "_Q"][b]) <= 4 * n * eps * nrm * np.linalg.norm(W)
        assert lu_backward_error(A[b], LU[b], ipiv[b]) / (n * eps) < 10


def test_getrs_large_golden(handle):
    A = uniform_general(256, 256, 2, seed=1256)
    B = np.random.default_rng(1257).uniform(-1, 1, (2, 256, 4))
    dA, dB = dev(to_colmajor(A)), dev(to_colmajor(B))
    dP = dev(np.zeros(2 * 256, np.int32))
    dI = dev(np.full(2, -1, np.int32))
    st = rs.call("rocsolver_dgesv_strided_batched", handle, 256, 4, ptr(dA), 256, 256 * 256,
                 ptr(dP), 256, ptr(dB), 256, 256 * 4, ptr(dI), 2)
    assert st == rs.SUCCESS
    np.testing.assert_array_equal(host(dP).reshape(2, 256), GOLD["bigrf_uni_n256_ipiv"])
    X = from_colmajor(host(dB), 2, 256, 4, 256, 256 * 4)
    eps = eps_of(np.float64)
    for b in range(2):
        kappa = np.linalg.cond(A[b], np.inf)
        d = np.abs(X[b] - GOLD["bigrs_uni_n256_r4_X"][b]).max()
        assert d <= 256 * eps * kappa * np.abs(X[b]).max()
        assert solve_backward_error(A[b], X[b], B[b]) < 10 * 256 * eps


# -------------------------------------------- the mixed-precision configuration's inputs
def test_getrf_pivots_on_cond_graded_config_inputs(handle):
    """Plain dgetrf on the first 256 members of the benchmark's n = 256 cond-graded batch
    (cond(A) log-uniform in [1e1, 1e6], the same generator and seed as the benchmark):
    ipiv and info exactly the oracle's, backward error < 10."""
    import torch
    from bench import make_cond_matrices
    A = make_cond_matrices(torch, 256, 256, seed=2, device=torch.device("cuda")).cpu().numpy()
    LU, ipiv, info = _getrf(handle, A)
    flat = to_colmajor(A)
    oP, oI = np.zeros(256 * 256, np.int32), np.zeros(256, np.int32)
    oracle.getrf(256, 256, flat, 256, 256 * 256, oP, 256, oI, 256, nthreads=NT)
    np.testing.assert_array_equal(info, oI)
    np.testing.assert_array_equal(ipiv, oP.reshape(256, 256))
    eps = eps_of(np.float64)
    for b in range(0, 256, 8):
        assert lu_backward_error(A[b], LU[b], ipiv[b]) / (256 * eps) < 10


# ------------------------------------------------------ variable-size configuration shape
def test_gesv_vbatched_config_shape(handle):
    """rocsolver_dgesv_vbatched on 256 members drawn like the variable-size configuration
    (n ~ U[8, 512] with n = 512 present, nrhs ~ U[1, 16], A ~ U[-1,1] + 0.1 n I, members in
    512 x 512 slots with lda = 512, max_n = 512, max_nrhs = 16: the tuning table's n_max 512
    entry): ipiv and info exactly the oracle's for every member, backward error < 10."""
    import torch
    rng = np.random.default_rng(44)
    bc, nmax = 256, 512
    ns = rng.integers(8, nmax + 1, bc)
    ns[7], ns[100] = 512, 8
    ks = rng.integers(1, 17, bc)
    A = rng.uniform(-1, 1, (bc, nmax, nmax))
    A += 0.1 * ns[:, None, None] * np.eye(nmax)[None]
    B = rng.uniform(-1, 1, (bc, 16, nmax))           # member b: column-major nmax x 16
    dA = torch.from_numpy(A.transpose(0, 2, 1).copy()).cuda()  # column-major, lda = nmax
    dB = torch.from_numpy(B.copy()).cuda()
    dP = torch.zeros(bc * nmax, dtype=torch.int32, device="cuda")
    dI = torch.full((bc,), -9, dtype=torch.int32, device="cuda")
    ar = torch.arange(bc, device="cuda", dtype=torch.int64)
    pa = ar * (nmax * nmax * 8) + dA.data_ptr()
    pb = ar * (16 * nmax * 8) + dB.data_ptr()
    pp = ar * (nmax * 4) + dP.data_ptr()
    dn = torch.from_numpy(ns.astype(np.int32)).cuda()
    dk = torch.from_numpy(ks.astype(np.int32)).cuda()
    ld = torch.full((bc,), nmax, dtype=torch.int32, device="cuda")
    st = rs.call("rocsolver_dgesv_vbatched", handle, ptr(dn), ptr(dk), ptr(pa), ptr(ld), ptr(pp),
                 ptr(pb), ptr(ld), ptr(dI), nmax, 16, bc)
    assert st == rs.SUCCESS
    X = host(dB)
    P = host(dP).reshape(bc, nmax)
    info = host(dI)
    assert not info.any()
    # oracle, per member (one call per member; members grouped to use all host threads)
    eps = eps_of(np.float64)
    for b in range(bc):
        n, k = int(ns[b]), int(ks[b])
        oA = A[b, :n, :n].T.copy().reshape(-1)
        oB = B[b, :k, :n].copy().reshape(-1)
        oP, oI = np.zeros(n, np.int32), np.zeros(1, np.int32)
        oracle.gesv(n, k, oA, n, n * n, oP, n, oB, n, n * k, oI, 1)
        assert oI[0] == info[b]
        np.testing.assert_array_equal(P[b, :n], oP, err_msg=f"member {b} n={n}")
        xb = X[b, :k, :n].T
        be = solve_backward_error(A[b, :n, :n], xb, B[b, :k, :n].T)
        assert be < 10 * n * eps, (b, n, be)


# ---------------------------------------------------------------- non-batched entry points
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [7, 32, 100, 256])
def test_nonbatched_lu_family(handle, dtype, n):
    """rocsolver_{s,d}getrf, getrs (N and T) and gesv on one matrix with lda = ldb = n + 3:
    ipiv and info exactly the oracle's, the padding rows untouched."""
    p = prefix(dtype)
    eps = eps_of(dtype)
    lda = n + 3
    A = uniform_general(n, n, 1, seed=900 + n).astype(dtype)
    B = uniform_general(n, 2, 1, seed=901 + n).astype(dtype)
    fA = to_colmajor(A, lda)
    dA = dev(fA)
    dP = dev(np.full(n, -1, np.int32))
    dI = dev(np.full(1, -1, np.int32))
    assert rs.call(f"rocsolver_{p}getrf", handle, n, n, ptr(dA), lda, ptr(dP), ptr(dI)) == rs.SUCCESS
    gA = host(dA)
    oA = to_colmajor(A)
    oP, oI = np.zeros(n, np.int32), np.zeros(1, np.int32)
    oracle.getrf(n, n, oA, n, n * n, oP, n, oI, 1)
    np.testing.assert_array_equal(host(dP), oP)
    np.testing.assert_array_equal(host(dI), oI)
    assert np.isnan(gA.reshape(n, lda)[:, n:]).all()
    LU = from_colmajor(gA, 1, n, n, lda, lda * n)[0]
    for trans in (0, 1):
        dB = dev(to_colmajor(B, lda))
        op = rs.OP_T if trans else rs.OP_N
        assert rs.call(f"rocsolver_{p}getrs", handle, op, n, 2, ptr(dA), lda, ptr(dP), ptr(dB),
                       lda) == rs.SUCCESS
        X = from_colmajor(host(dB), 1, n, 2, lda, lda * 2)[0]
        opA = A[0].T if trans else A[0]
        assert solve_backward_error(opA.astype(np.float64), X.astype(np.float64),
                                    B[0].astype(np.float64)) < 10 * n * eps
    dA2, dB2 = dev(to_colmajor(A, lda)), dev(to_colmajor(B, lda))
    dP2, dI2 = dev(np.full(n, -1, np.int32)), dev(np.full(1, -1, np.int32))
    assert rs.call(f"rocsolver_{p}gesv", handle, n, 2, ptr(dA2), lda, ptr(dP2), ptr(dB2), lda,
                   ptr(dI2)) == rs.SUCCESS
    np.testing.assert_array_equal(host(dP2), oP)
    np.testing.assert_array_equal(host(dI2), 0)
    X = from_colmajor(host(dB2), 1, n, 2, lda, lda * 2)[0]
    assert solve_backward_error(A[0].astype(np.float64), X.astype(np.float64),
                                B[0].astype(np.float64)) < 10 * n * eps
    np.testing.assert_array_equal(from_colmajor(host(dA2), 1, n, n, lda, lda * n)[0], LU)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [5, 64, 130])
@pytest.mark.parametrize("lower", [True, False])
def test_nonbatched_cholesky_family(handle, dtype, n, lower):
    """rocsolver_{s,d}potrf, potrs and posv on one SPD matrix (and posv on a non-SPD one:
    info > 0 and B unchanged), lda = ldb = n + 2."""
    p = prefix(dtype)
    eps = eps_of(dtype)
    uplo = rs.FILL_LOWER if lower else rs.FILL_UPPER
    lda = n + 2
    A = spd_gram(n, 1, seed=70 + n).astype(dtype)
    B = uniform_general(n, 3, 1, seed=71 + n).astype(dtype)
    dA, dI = dev(to_colmajor(A, lda)), dev(np.full(1, -1, np.int32))
    assert rs.call(f"rocsolver_{p}potrf", handle, uplo, n, ptr(dA), lda, ptr(dI)) == rs.SUCCESS
    assert host(dI)[0] == 0
    C = from_colmajor(host(dA), 1, n, n, lda, lda * n)
    oA, oI = to_colmajor(A), np.zeros(1, np.int32)
    oracle.potrf(not lower, n, oA, n, n * n, oI, 1)
    oC = from_colmajor(oA, 1, n, n, n, n * n)
    tri = np.tril if lower else np.triu
    assert np.abs(tri(C[0]) - tri(oC[0])).max() <= 8 * n * eps * np.abs(oC[0]).max()
    dB = dev(to_colmajor(B, lda))
    assert rs.call(f"rocsolver_{p}potrs", handle, uplo, n, 3, ptr(dA), lda, ptr(dB),
                   lda) == rs.SUCCESS
    X = from_colmajor(host(dB), 1, n, 3, lda, lda * 3)[0]
    assert solve_backward_error(A[0].astype(np.float64), X.astype(np.float64),
                                B[0].astype(np.float64)) < 10 * n * eps
    for spd in (True, False):
        M = A.copy()
        if not spd:
            M[0, n // 2, n // 2] = -1.0
        dA2, dB2 = dev(to_colmajor(M, lda)), dev(to_colmajor(B, lda))
        dI2 = dev(np.full(1, -1, np.int32))
        assert rs.call(f"rocsolver_{p}posv", handle, uplo, n, 3, ptr(dA2), lda, ptr(dB2), lda,
                       ptr(dI2)) == rs.SUCCESS
        oM, oB, oI2 = to_colmajor(M), to_colmajor(B), np.zeros(1, np.int32)
        oracle.posv(not lower, n, 3, oM, n, n * n, oB, n, n * 3, oI2, 1)
        assert host(dI2)[0] == oI2[0]
        X = from_colmajor(host(dB2), 1, n, 3, lda, lda * 3)[0]
        if spd:
            assert oI2[0] == 0
            assert solve_backward_error(A[0].astype(np.float64), X.astype(np.float64),
                                        B[0].astype(np.float64)) < 10 * n * eps
        else:
            assert oI2[0] > 0
            np.testing.assert_array_equal(X, B[0])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [16, 64, 200])
def test_posv_batched_pointer_array(handle, dtype, n):
    """rocsolver_{s,d}posv_batched (pointer arrays), one failing member: info exactly the
    oracle's, the failing member's B unchanged, the others' backward error < 10."""
    p = prefix(dtype)
    eps = eps_of(dtype)
    bc, nrhs = 5, 4
    A = spd_gram(n, bc, seed=80 + n).astype(dtype)
    A[3, 1, 1] = -2.0
    B = np.random.default_rng(81 + n).standard_normal((bc, n, nrhs)).astype(dtype)
    dA, dB = dev(to_colmajor(A)), dev(to_colmajor(B))
    aA, aB = ptr_array(dA, bc, n * n), ptr_array(dB, bc, n * nrhs)
    dI = dev(np.full(bc, -1, np.int32))
    st = rs.call(f"rocsolver_{p}posv_batched", handle, rs.FILL_LOWER, n, nrhs, ptr(aA), n,
                 ptr(aB), n, ptr(dI), bc)
    assert st == rs.SUCCESS
    info = host(dI)
    X = from_colmajor(host(dB), bc, n, nrhs, n, n * nrhs)
    oA, oB, oI = to_colmajor(A), to_colmajor(B), np.zeros(bc, np.int32)
    oracle.posv(False, n, nrhs, oA, n, n * n, oB, n, n * nrhs, oI, bc)
    np.testing.assert_array_equal(info, oI)
    for b in range(bc):
        if info[b]:
            np.testing.assert_array_equal(X[b], B[b])
        else:
            assert solve_backward_error(A[b].astype(np.float64), X[b].astype(np.float64),
                                        B[b].astype(np.float64)) < 10 * n * eps
