"""The FP32 LU with its trailing update on the 5th-generation tensor cores (tcgen05: split-TF32
operands in shared memory, FP32 accumulators in tensor memory), selected per size class by a
tuning entry with fold = 2.  Every compiled tcgen05 variant is forced in turn through
rocsolver_b200_tuning_set and checked on rocsolver_sgetrf_tf32_strided_batched: info exactly
the oracle's (never the negative value that reports an expired tensor-core wait), the
FP32-level backward error ||PA - LU||_F / (n ||A||_F eps32) < 10 with the returned pivots,
the oracle's pivots except where FP32 rounding flips a near tie (< 2 %), rectangular shapes,
a singular member, and the mixed-precision solver running on it."""
import numpy as np
import pytest

import rocsolver_b200 as rs
from tests.gpu_util import GpuHandle, dev, host, ptr
from tests.norms import eps_of, lu_backward_error, solve_backward_error
from tests.refcases import cond_graded, from_colmajor, to_colmajor, uniform_general
from tests.test_lu_gpu import oracle_getrf

pytestmark = pytest.mark.gpu

# (threads, rows per thread, panel width) of the compiled tcgen05 variants
UM_VARIANTS = [(128, 1, 32), (128, 2, 32), (256, 1, 32), (256, 2, 32), (256, 2, 16),
               (256, 4, 16), (256, 4, 8), (256, 8, 8)]


@pytest.fixture(scope="module")
def handle():
    h = GpuHandle()
    yield h.value
    h.close()


@pytest.fixture
def restore_table():
    old = rs.tuning_table()
    yield
    assert rs.set_tuning_table(old) == rs.SUCCESS


def sgetrf_tf32(handle, A):
    bc, m, n = A.shape
    mn = min(m, n)
    dA = dev(to_colmajor(A))
    dP = dev(np.full(bc * mn, -7, np.int32))
    dI = dev(np.full(bc, -7, np.int32))
    st = rs.call("rocsolver_sgetrf_tf32_strided_batched", handle, m, n, ptr(dA), m, m * n,
                 ptr(dP), mn, ptr(dI), bc)
    assert st == rs.SUCCESS, rs.STATUS_NAMES[st]
    return from_colmajor(host(dA), bc, m, n, m, m * n), host(dP).reshape(bc, mn), host(dI)


CASES = []
for nt, r, jb in UM_VARIANTS:
    cap = nt * r
    for n in sorted({min(cap, 300), cap, cap // 2 + 5}):
        for cw in (64, 128):
            CASES.append((nt, r, jb, n, cw))


@pytest.mark.parametrize("nt,r,jb,n,cw", CASES)
def test_forced_umma_variant(handle, restore_table, nt, r, jb, n, cw):
    assert rs.set_tuning_table(f"getrf t {n} {nt} {r} {jb} {cw} 2\n") == rs.SUCCESS
    bc = 3
    A = uniform_general(n, n, bc, seed=5000 + n + jb).astype(np.float32)
    LU, ipiv, info = sgetrf_tf32(handle, A)
    _, oipiv, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(info, oinfo)
    for b in range(bc):
        be = lu_backward_error(A[b].astype(np.float64), LU[b].astype(np.float64), ipiv[b])
        assert be / (n * eps_of(np.float32)) < 10, (b, be)
    if n <= 512:
        assert (ipiv != oipiv).mean() < 0.02


@pytest.mark.parametrize("m,n", [(300, 120), (120, 300), (512, 64), (257, 257)])
def test_umma_rectangular_and_singular(handle, restore_table, m, n):
    assert rs.set_tuning_table(f"getrf t {max(m, 512)} 256 2 32 128 2\n") == rs.SUCCESS
    A = uniform_general(m, n, 3, seed=m * 7 + n).astype(np.float32)
    A[1][:, min(m, n) // 2] = 0.0
    LU, ipiv, info = sgetrf_tf32(handle, A)
    _, _, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(info, oinfo)
    assert info[1] != 0 and info[0] == 0
    mn = min(m, n)
    for b in (0, 2):
        L = np.tril(LU[b][:, :mn].astype(np.float64), -1) + np.eye(m, mn)
        U = np.triu(LU[b][:mn, :].astype(np.float64))
        PA = A[b].astype(np.float64).copy()
        for k in range(mn):
            p = ipiv[b][k] - 1
            if p != k:
                PA[[k, p]] = PA[[p, k]]
        err = np.linalg.norm(PA - L @ U) / np.linalg.norm(A[b])
        assert err / (max(m, n) * eps_of(np.float32)) < 10


@pytest.mark.parametrize("n,cfg", [(256, "128 2 32 64"), (256, "256 1 32 64"),
                                   (512, "256 2 32 128"), (1024, "256 4 16 128")])
def test_dsgesv_on_umma_lu(handle, restore_table, n, cfg):
    """The mixed-precision solver with its FP32 factorisation on tcgen05: every member
    reaches FP64 backward error <= 1e-13 (refinement converges, no FP64 fallback)."""
    assert rs.set_tuning_table(f"getrf t {n} {cfg} 2\n") == rs.SUCCESS
    bc = 8
    A = cond_graded(n, bc, seed=600 + n, lo=1.0, hi=5.0)
    B = np.random.default_rng(n).uniform(-1, 1, (bc, n, 1))
    dA, dB = dev(to_colmajor(A)), dev(to_colmajor(B))
    dX = dev(np.zeros(bc * n))
    dP = dev(np.zeros(bc * n, np.int32))
    dI = dev(np.full(bc, -1, np.int32))
    dT = dev(np.full(bc, -99, np.int32))
    st = rs.call("rocsolver_dsgesv_strided_batched", handle, n, 1, ptr(dA), n, n * n, ptr(dP),
                 n, ptr(dB), n, n, ptr(dX), n, n, ptr(dT), ptr(dI), bc)
    assert st == rs.SUCCESS
    it, info = host(dT), host(dI)
    assert not info.any()
    assert np.all(it >= 0), it
    X = from_colmajor(host(dX), bc, n, 1, n, n)
    for b in range(bc):
        assert solve_backward_error(A[b], X[b], B[b]) <= 1e-13


# ---- two-level LU (fold = 3): outer panels of 64 columns factored by the one-level kernel
# body, one K = 64 tcgen05 trailing update per outer panel
LU2_VARIANTS = [(256, 2, 32), (256, 2, 16), (256, 4, 16), (256, 4, 8), (256, 8, 8)]
LU2_CASES = []
for nt, r, jb in LU2_VARIANTS:
    cap = nt * r
    for n in sorted({min(cap, 300), cap, 200, 65}):
        LU2_CASES.append((nt, r, jb, n, 128 if n >= 128 else 64))


@pytest.mark.parametrize("nt,r,jb,n,cw", LU2_CASES)
def test_forced_two_level_variant(handle, restore_table, nt, r, jb, n, cw):
    assert rs.set_tuning_table(f"getrf t {n} {nt} {r} {jb} {cw} 3\n") == rs.SUCCESS
    bc = 2 if n > 1024 else 3
    A = uniform_general(n, n, bc, seed=7000 + n + jb).astype(np.float32)
    LU, ipiv, info = sgetrf_tf32(handle, A)
    _, oipiv, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(info, oinfo)
    for b in range(bc):
        be = lu_backward_error(A[b].astype(np.float64), LU[b].astype(np.float64), ipiv[b])
        assert be / (n * eps_of(np.float32)) < 10, (b, be)
    if n <= 512:
        assert (ipiv != oipiv).mean() < 0.02


@pytest.mark.parametrize("m,n", [(300, 120), (120, 300), (512, 64), (257, 257), (400, 130)])
def test_two_level_rectangular_and_singular(handle, restore_table, m, n):
    assert rs.set_tuning_table("getrf t 512 256 2 32 128 3\n") == rs.SUCCESS
    A = uniform_general(m, n, 3, seed=m * 11 + n).astype(np.float32)
    A[1][:, min(m, n) // 2 + 3] = 0.0
    LU, ipiv, info = sgetrf_tf32(handle, A)
    _, _, oinfo = oracle_getrf(A)
    np.testing.assert_array_equal(info, oinfo)
    assert info[1] != 0 and info[0] == 0
    mn = min(m, n)
    for b in (0, 2):
        L = np.tril(LU[b][:, :mn].astype(np.float64), -1) + np.eye(m, mn)
        U = np.triu(LU[b][:mn, :].astype(np.float64))
        PA = A[b].astype(np.float64).copy()
        for k in range(mn):
            p = ipiv[b][k] - 1
            if p != k:
                PA[[k, p]] = PA[[p, k]]
        err = np.linalg.norm(PA - L @ U) / np.linalg.norm(A[b])
        assert err / (max(m, n) * eps_of(np.float32)) < 10


@pytest.mark.parametrize("n,cfg", [(512, "256 2 32 128"), (1024, "256 4 16 128")])
def test_dsgesv_on_two_level_lu(handle, restore_table, n, cfg):
    assert rs.set_tuning_table(f"getrf t {n} {cfg} 3\n") == rs.SUCCESS
    bc = 4
    A = cond_graded(n, bc, seed=800 + n, lo=1.0, hi=5.0)
    B = np.random.default_rng(n + 1).uniform(-1, 1, (bc, n, 1))
    dA, dB = dev(to_colmajor(A)), dev(to_colmajor(B))
    dX = dev(np.zeros(bc * n))
    dP = dev(np.zeros(bc * n, np.int32))
    dI = dev(np.full(bc, -1, np.int32))
    dT = dev(np.full(bc, -99, np.int32))
    st = rs.call("rocsolver_dsgesv_strided_batched", handle, n, 1, ptr(dA), n, n * n, ptr(dP),
                 n, ptr(dB), n, n, ptr(dX), n, n, ptr(dT), ptr(dI), bc)
    assert st == rs.SUCCESS
    it, info = host(dT), host(dI)
    assert not info.any()
    X = from_colmajor(host(dX), bc, n, 1, n, n)
    for b in range(bc):
        assert solve_backward_error(A[b], X[b], B[b]) <= 1e-13
