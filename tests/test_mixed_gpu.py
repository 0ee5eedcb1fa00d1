"""GPU tests of the mixed-precision solver rocsolver_dsgesv_strided_batched (FP32 LU,
FP64 iterative refinement, FP64 fallback), against the FP64 oracle solution and the
LAPACK dsgesv contract (iter codes, A/B/X/ipiv/info behaviour)."""
import ctypes

import numpy as np
import pytest

import oracle
import rocsolver_b200 as rs
from tests.gpu_util import GpuHandle, dev, host, ptr
from tests.norms import solve_backward_error
from tests.refcases import from_colmajor, to_colmajor, uniform_general

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    h = GpuHandle()
    yield h.value
    h.close()


def cond_matrices(n, bc, seed, lo=1.0, hi=6.0):
    rng = np.random.default_rng(seed)
    out = np.empty((bc, n, n))
    for b in range(bc):
        U, _ = np.linalg.qr(rng.standard_normal((n, n)))
        V, _ = np.linalg.qr(rng.standard_normal((n, n)))
        lk = rng.uniform(lo, hi)
        s = 10.0 ** (-lk * np.linspace(0, 1, n))
        out[b] = (U * s) @ V.T
    return out


def gpu_dsgesv(handle, A, B, ldx=None):
    bc, n, _ = A.shape
    nrhs = B.shape[2]
    ldx = n if ldx is None else ldx
    dA = dev(to_colmajor(A))
    dB = dev(to_colmajor(B))
    dX = dev(np.full(bc * ldx * nrhs, np.nan))
    dP = dev(np.zeros(bc * n, np.int32))
    dI = dev(np.full(bc, -9, np.int32))
    dT = dev(np.full(bc, -99, np.int32))
    st = rs.call("rocsolver_dsgesv_strided_batched", handle, n, nrhs, ptr(dA), n, n * n, ptr(dP),
                 n, ptr(dB), n, n * nrhs, ptr(dX), ldx, ldx * nrhs, ptr(dT), ptr(dI), bc)
    assert st == rs.SUCCESS, rs.STATUS_NAMES[st]
    return (from_colmajor(host(dA), bc, n, n, n, n * n), host(dP).reshape(bc, n),
            from_colmajor(host(dB), bc, n, nrhs, n, n * nrhs),
            from_colmajor(host(dX), bc, n, nrhs, ldx, ldx * nrhs), host(dT), host(dI))


def oracle_x(A, B):
    bc, n, _ = A.shape
    nrhs = B.shape[2]
    oA, oB = to_colmajor(A), to_colmajor(B)
    oP, oI = np.zeros(bc * n, np.int32), np.zeros(bc, np.int32)
    oracle.gesv(n, nrhs, oA, n, n * n, oP, n, oB, n, n * nrhs, oI, bc, nthreads=8)
    return from_colmajor(oB, bc, n, nrhs, n, n * nrhs), oI


@pytest.mark.parametrize("n,bc,nrhs", [(256, 24, 1), (100, 16, 3), (32, 64, 1), (17, 40, 5),
                                       (512, 4, 2)])
def test_dsgesv_converges_to_fp64_accuracy(handle, n, bc, nrhs):
    """cond(A) log-uniform in [1e1, 1e6]: refinement converges (iter >= 0, <= 10), backward
    error <= 1e-13 per member (computed in long double), A and B unchanged, ipiv = FP32
    pivots of the oracle's LU of float32(A)."""
    A = cond_matrices(n, bc, seed=n + bc)
    B = np.random.default_rng(n).uniform(-1, 1, (bc, n, nrhs))
    A2, ipiv, B2, X, it, info = gpu_dsgesv(handle, A, B)
    assert np.all(info == 0)
    assert np.all(it >= 0) and np.all(it <= 10), it
    np.testing.assert_array_equal(A2, A)
    np.testing.assert_array_equal(B2, B)
    OX, _ = oracle_x(A, B)
    for b in range(bc):
        be = solve_backward_error(A[b], X[b], B[b])
        assert be <= 1e-13, (b, be)
        kappa = np.linalg.cond(A[b], np.inf)
        fe = np.abs(X[b] - OX[b]).max() / np.abs(OX[b]).max()
        assert fe <= 50 * kappa * 1.1e-16 + 1e-15, (b, fe, kappa)
    # pivots are those of the FP32 factorisation.  FP32 rounding differs from the oracle's
    # FP32 LU (the device fuses multiply-adds and forms U12 with the inverse of L11), which
    # flips near-tied pivots in late columns of these graded matrices: allow < 1%
    A32 = A.astype(np.float32)
    flat = to_colmajor(A32)
    oP, oI = np.zeros(bc * n, np.int32), np.zeros(bc, np.int32)
    oracle.getrf(n, n, flat, n, n * n, oP, n, oI, bc, nthreads=8)
    mism = (ipiv != oP.reshape(bc, n)).mean()
    assert mism < 0.01, mism


def test_dsgesv_fallback_ill_conditioned(handle):
    """cond ~ 1e12: FP32 refinement cannot converge -> iter = -11, FP64 re-solve: A holds
    the FP64 LU, ipiv/info are FP64's, X matches the FP64 oracle."""
    n, bc = 64, 6
    A = cond_matrices(n, bc, seed=5, lo=11.5, hi=12.5)
    B = np.random.default_rng(1).uniform(-1, 1, (bc, n, 1))
    A2, ipiv, _, X, it, info = gpu_dsgesv(handle, A, B)
    assert np.all(it < 0), it
    assert np.all(info == 0)
    oA = to_colmajor(A)
    oP, oI = np.zeros(bc * n, np.int32), np.zeros(bc, np.int32)
    oracle.getrf(n, n, oA, n, n * n, oP, n, oI, bc)
    np.testing.assert_array_equal(ipiv, oP.reshape(bc, n))
    from tests.norms import lu_backward_error
    for b in range(bc):
        # cond ~ 1e12: compare the FP64 factors by backward error, not entrywise
        assert lu_backward_error(A[b], A2[b], ipiv[b]) / (n * 2.2e-16) < 10
        be = solve_backward_error(A[b], X[b], B[b])
        assert be < 1e-14


def test_dsgesv_mixed_batch_codes(handle):
    """One batch mixing: converging members, an FP32-overflow member (-2), an exactly
    singular member (FP32 LU singular -> -3 -> FP64 info > 0, X not computed), and an
    ill-conditioned member (-11)."""
    n, bc = 48, 6
    A = cond_matrices(n, bc, seed=9)
    A[1, 3, 4] = 1e39                       # overflows FP32
    A[2, :, 7] = 0.0                        # singular in both precisions
    A[3] = cond_matrices(n, 1, seed=11, lo=12.0, hi=12.0)[0]
    B = np.random.default_rng(2).uniform(-1, 1, (bc, n, 2))
    A2, ipiv, B2, X, it, info = gpu_dsgesv(handle, A, B)
    assert it[0] >= 0 and it[4] >= 0 and it[5] >= 0
    assert it[1] == -2 and it[2] == -3 and it[3] == -11, it
    assert info[2] == 8 and info[0] == 0 and info[1] == 0 and info[3] == 0
    np.testing.assert_array_equal(B2, B)
    for b in (0, 1, 3, 4, 5):
        be = solve_backward_error(A[b], X[b], B[b])
        assert be < 1e-13, (b, be)
    for b in (0, 4, 5):
        np.testing.assert_array_equal(A2[b], A[b])


def test_dsgesv_quick_return_and_workspace(handle):
    dI = dev(np.full(3, 7, np.int32))
    dT = dev(np.full(3, 7, np.int32))
    st = rs.call("rocsolver_dsgesv_strided_batched", handle, 0, 1, None, 1, 1, None, 1, None, 1,
                 1, None, 1, 1, ptr(dT), ptr(dI), 3)
    assert st == rs.SUCCESS
    np.testing.assert_array_equal(host(dI), 0)
    np.testing.assert_array_equal(host(dT), 0)
    # size query reports the FP32 copy of A as workspace
    sz = ctypes.c_size_t()
    f = ctypes.c_void_p(0x1000)
    assert rs.call("rocblas_start_device_memory_size_query", handle) == rs.SUCCESS
    st = rs.call("rocsolver_dsgesv_strided_batched", handle, 64, 1, f, 64, 4096, f, 64, f, 64, 64,
                 f, 64, 64, f, f, 10)
    assert st == rs.SIZE_INCREASED
    rs.call("rocblas_stop_device_memory_size_query", handle, ctypes.byref(sz))
    assert sz.value >= 64 * 64 * 4 * 10


def test_dsgesv_user_workspace_too_small():
    import torch
    h = rs.Handle(torch.cuda.current_stream().cuda_stream)
    try:
        buf = torch.empty(1024, dtype=torch.uint8, device="cuda")
        assert rs.call("rocblas_set_workspace", h.value, ptr(buf), 1024) == rs.SUCCESS
        A = uniform_general(64, 64, 4, seed=1) + 8 * np.eye(64)[None]
        dA = dev(to_colmajor(A))
        dB = dev(np.ones(64 * 4))
        dX = dev(np.zeros(64 * 4))
        dP = dev(np.zeros(64 * 4, np.int32))
        dI = dev(np.zeros(4, np.int32))
        dT = dev(np.zeros(4, np.int32))
        st = rs.call("rocsolver_dsgesv_strided_batched", h.value, 64, 1, ptr(dA), 64, 4096,
                     ptr(dP), 64, ptr(dB), 64, 64, ptr(dX), 64, 64, ptr(dT), ptr(dI), 4)
        assert st == rs.MEMORY_ERROR
        big = torch.empty(1 << 22, dtype=torch.uint8, device="cuda")
        assert rs.call("rocblas_set_workspace", h.value, ptr(big), 1 << 22) == rs.SUCCESS
        st = rs.call("rocsolver_dsgesv_strided_batched", h.value, 64, 1, ptr(dA), 64, 4096,
                     ptr(dP), 64, ptr(dB), 64, 64, ptr(dX), 64, 64, ptr(dT), ptr(dI), 4)
        assert st == rs.SUCCESS
        assert np.all(host(dT) >= 0)
    finally:
        h.close()
