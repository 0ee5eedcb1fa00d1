"""GPU tests of the batched-solve adjoint (rocsolver_{s,d}getrs_adjoint_strided_batched,
rocsolver_{s,d}potrs_adjoint_strided_batched): against an explicit host-LAPACK reference
gradient (gB = A^{-T} G, gA = -gB X^T), central finite differences (FP64, h = 1e-6), and
torch.autograd.gradcheck through a test-only autograd wrapper of the C-ABI calls."""
import numpy as np
import pytest

import rocsolver_b200 as rs
from tests.gpu_util import GpuHandle, dev, host, prefix, ptr
from tests.refcases import from_colmajor, spd_gram, to_colmajor

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    h = GpuHandle()
    yield h.value
    h.close()


def forward_lu(handle, A, B):
    """getrf + getrs on the GPU; returns device buffers (LU, ipiv, X)."""
    bc, n, _ = A.shape
    nrhs = B.shape[2]
    p = prefix(A.dtype)
    dA = dev(to_colmajor(A))
    dX = dev(to_colmajor(B))
    dP = dev(np.zeros(bc * n, np.int32))
    dI = dev(np.zeros(bc, np.int32))
    rs.check(rs.call(f"rocsolver_{p}getrf_strided_batched", handle, n, n, ptr(dA), n, n * n,
                     ptr(dP), n, ptr(dI), bc), "getrf")
    rs.check(rs.call(f"rocsolver_{p}getrs_strided_batched", handle, rs.OP_N, n, nrhs, ptr(dA), n,
                     n * n, ptr(dP), n, ptr(dX), n, n * nrhs, bc), "getrs")
    assert not host(dI).any()
    return dA, dP, dX


def adjoint_lu(handle, dA, dP, dX, G):
    bc, n, nrhs = G.shape
    p = prefix(G.dtype)
    dG = dev(to_colmajor(G))
    dgA = dev(np.full(bc * n * n, np.nan, G.dtype))
    dgB = dev(np.full(bc * n * nrhs, np.nan, G.dtype))
    rs.check(rs.call(f"rocsolver_{p}getrs_adjoint_strided_batched", handle, n, nrhs, ptr(dA), n,
                     n * n, ptr(dP), n, ptr(dX), n, n * nrhs, ptr(dG), n, n * nrhs, ptr(dgA), n,
                     n * n, ptr(dgB), n, n * nrhs, bc), "getrs_adjoint")
    return (from_colmajor(host(dgA), bc, n, n, n, n * n),
            from_colmajor(host(dgB), bc, n, nrhs, n, n * nrhs))


def reference_grad(A, B, G):
    A64, B64, G64 = A.astype(np.float64), B.astype(np.float64), G.astype(np.float64)
    X = np.linalg.solve(A64, B64)
    gB = np.linalg.solve(A64.transpose(0, 2, 1), G64)
    gA = -gB @ X.transpose(0, 2, 1)
    return gA, gB, X


def c5_inputs(n, bc, nrhs, dtype, seed):
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, (bc, n, n)) + 4.0 * np.eye(n)[None]
    B = rng.standard_normal((bc, n, nrhs))
    G = rng.standard_normal((bc, n, nrhs))
    return A.astype(dtype), B.astype(dtype), G.astype(dtype)


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-11), (np.float32, 2e-4)])
@pytest.mark.parametrize("n,nrhs", [(128, 8), (5, 3), (33, 1), (70, 12)])
def test_getrs_adjoint_vs_reference_gradient(handle, dtype, tol, n, nrhs):
    """Adjoint configuration shape (n=128, nrhs=8, A = U[-1,1] + 4 I, B, G ~ N(0,1)) on a
    batch of 32, plus edge shapes; relative error against the explicit reference."""
    A, B, G = c5_inputs(n, 32, nrhs, dtype, seed=n + nrhs)
    dA, dP, dX = forward_lu(handle, A, B)
    gA, gB = adjoint_lu(handle, dA, dP, dX, G)
    rgA, rgB, _ = reference_grad(A, B, G)
    eA = np.abs(gA - rgA).max() / np.abs(rgA).max()
    eB = np.abs(gB - rgB).max() / np.abs(rgB).max()
    assert eA < tol and eB < tol, (eA, eB)


def test_getrs_adjoint_central_differences(handle):
    """dL/dA and dL/dB for L = <G, X(A, B)> by central differences (FP64, h = 1e-6) at
    sampled entries, against the GPU adjoint."""
    n, nrhs = 24, 3
    A, B, G = c5_inputs(n, 2, nrhs, np.float64, seed=3)
    dA, dP, dX = forward_lu(handle, A, B)
    gA, gB = adjoint_lu(handle, dA, dP, dX, G)
    h = 1e-6
    rng = np.random.default_rng(0)

    def loss(Ab, Bb, Gb):
        return float((Gb * np.linalg.solve(Ab, Bb)).sum())
    worst = 0.0
    for b in range(2):
        for _ in range(12):
            i, j = rng.integers(0, n, 2)
            Ap, Am = A[b].copy(), A[b].copy()
            Ap[i, j] += h
            Am[i, j] -= h
            fd = (loss(Ap, B[b], G[b]) - loss(Am, B[b], G[b])) / (2 * h)
            worst = max(worst, abs(fd - gA[b, i, j]) / max(1.0, abs(fd)))
            k, c = rng.integers(0, n), rng.integers(0, nrhs)
            Bp, Bm = B[b].copy(), B[b].copy()
            Bp[k, c] += h
            Bm[k, c] -= h
            fd = (loss(A[b], Bp, G[b]) - loss(A[b], Bm, G[b])) / (2 * h)
            worst = max(worst, abs(fd - gB[b, k, c]) / max(1.0, abs(fd)))
    assert worst < 1e-7, worst


def test_getrs_adjoint_gradcheck(handle):
    """torch.autograd.gradcheck of X = solve(A, B) with forward = getrf + getrs and
    backward = the adjoint entry point (wrapper exists only here, in the tests)."""
    import torch

    class Solve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, A, B):
            bc, n, _ = A.shape
            nrhs = B.shape[2]
            dA = A.detach().transpose(1, 2).contiguous()
            dX = B.detach().transpose(1, 2).contiguous()
            dP = torch.zeros(bc * n, dtype=torch.int32, device=A.device)
            dI = torch.zeros(bc, dtype=torch.int32, device=A.device)
            rs.check(rs.call("rocsolver_dgetrf_strided_batched", handle, n, n, ptr(dA), n, n * n,
                             ptr(dP), n, ptr(dI), bc), "getrf")
            rs.check(rs.call("rocsolver_dgetrs_strided_batched", handle, rs.OP_N, n, nrhs,
                             ptr(dA), n, n * n, ptr(dP), n, ptr(dX), n, n * nrhs, bc), "getrs")
            ctx.save_for_backward(dA, dP, dX)
            return dX.transpose(1, 2).contiguous()

        @staticmethod
        def backward(ctx, gX):
            dA, dP, dX = ctx.saved_tensors
            bc, n, _ = dA.shape
            nrhs = dX.shape[1]
            dG = gX.transpose(1, 2).contiguous()
            gA = torch.empty(bc, n, n, dtype=torch.float64, device=dA.device)
            gB = torch.empty(bc, nrhs, n, dtype=torch.float64, device=dA.device)
            rs.check(rs.call("rocsolver_dgetrs_adjoint_strided_batched", handle, n, nrhs,
                             ptr(dA), n, n * n, ptr(dP), n, ptr(dX), n, n * nrhs, ptr(dG), n,
                             n * nrhs, ptr(gA), n, n * n, ptr(gB), n, n * nrhs, bc), "adjoint")
            torch.cuda.synchronize()
            return gA.transpose(1, 2), gB.transpose(1, 2)

    g = torch.Generator(device="cpu").manual_seed(0)
    A = (torch.rand(2, 6, 6, generator=g, dtype=torch.float64) * 2 - 1 + 4 * torch.eye(6)).cuda()
    B = torch.randn(2, 6, 2, generator=g, dtype=torch.float64).cuda()
    A.requires_grad_(True)
    B.requires_grad_(True)
    assert torch.autograd.gradcheck(Solve.apply, (A, B), eps=1e-6, atol=1e-8, rtol=1e-6)


@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-11), (np.float32, 2e-4)])
def test_potrs_adjoint(handle, lower, dtype, tol):
    n, nrhs, bc = 64, 4, 8
    A = spd_gram(n, bc, seed=4).astype(dtype)
    rng = np.random.default_rng(5)
    B = rng.standard_normal((bc, n, nrhs)).astype(dtype)
    G = rng.standard_normal((bc, n, nrhs)).astype(dtype)
    p = prefix(dtype)
    uplo = rs.FILL_LOWER if lower else rs.FILL_UPPER
    dA = dev(to_colmajor(A))
    dX = dev(to_colmajor(B))
    dI = dev(np.zeros(bc, np.int32))
    rs.check(rs.call(f"rocsolver_{p}potrf_strided_batched", handle, uplo, n, ptr(dA), n, n * n,
                     ptr(dI), bc), "potrf")
    rs.check(rs.call(f"rocsolver_{p}potrs_strided_batched", handle, uplo, n, nrhs, ptr(dA), n,
                     n * n, ptr(dX), n, n * nrhs, bc), "potrs")
    dG = dev(to_colmajor(G))
    dgA = dev(np.zeros(bc * n * n, dtype))
    rs.check(rs.call(f"rocsolver_{p}potrs_adjoint_strided_batched", handle, uplo, n, nrhs,
                     ptr(dA), n, n * n, ptr(dX), n, n * nrhs, ptr(dG), n, n * nrhs, ptr(dgA), n,
                     n * n, ptr(dG), n, n * nrhs, bc), "potrs_adjoint")  # gB aliases G
    gA = from_colmajor(host(dgA), bc, n, n, n, n * n)
    gB = from_colmajor(host(dG), bc, n, nrhs, n, n * nrhs)
    rgA, rgB, _ = reference_grad(A, B, G)
    assert np.abs(gA - rgA).max() / np.abs(rgA).max() < tol
    assert np.abs(gB - rgB).max() / np.abs(rgB).max() < tol
