"""Every configuration the tuning table can select gives the oracle's results: the CTA LU
variants (threads, rows per thread, panel width), chunk widths and interchange folding
are forced one at a time through rocsolver_b200_tuning_set, then getrf is compared with
the oracle (ipiv/info exact, factor error <= 4*min(m,n)*eps) and the variable-size gesv
with per-member LAPACK-style residual checks.  The active table is restored afterwards."""
import numpy as np
import pytest

import rocsolver_b200 as rs
from rocsolver_b200.tune import LU_VARIANTS, VB_VARIANTS
from tests.refcases import uniform_general
from tests.test_lu_gpu import check_getrf, gpu_getrf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    from tests.gpu_util import GpuHandle
    h = GpuHandle()
    yield h.value
    h.close()


@pytest.fixture
def restore_table():
    old = rs.tuning_table()
    yield
    assert rs.set_tuning_table(old) == rs.SUCCESS


CASES = []
for nt, r, jb in LU_VARIANTS:
    cap = nt * r
    for m, n in {(min(cap, 300), min(cap, 300)), (cap // 2 + 3, cap // 2 + 3),
                 (min(cap, 200), 70)}:
        if m > 32 and m <= cap:
            for cw, fold in ((32, 1), (64, 0), (128, 1)):
                CASES.append((nt, r, jb, m, n, cw, fold))


@pytest.mark.parametrize("nt,r,jb,m,n,cw,fold", CASES)
@pytest.mark.parametrize("prec", ["d", "s"])
def test_forced_getrf_config(handle, restore_table, nt, r, jb, m, n, cw, fold, prec):
    dtype = np.float64 if prec == "d" else np.float32
    assert rs.set_tuning_table(f"getrf {prec} {m} {nt} {r} {jb} {cw} {fold}\n") == rs.SUCCESS
    A = uniform_general(m, n, 3, seed=77 * m + n).astype(dtype)
    LU, ipiv, info, _ = gpu_getrf(handle, A)
    if prec == "d":
        check_getrf(A, LU, ipiv, info)
    else:
        # FP32 near-ties may pick a different pivot than the oracle: compare the factors'
        # backward error instead of the pivots
        from tests.norms import lu_backward_error
        assert np.all(info == 0)
        mn = min(m, n)
        for b in range(3):
            if m == n:
                be = lu_backward_error(A[b].astype(np.float64), LU[b].astype(np.float64),
                                       ipiv.reshape(3, mn)[b])
                assert be / (n * np.finfo(np.float32).eps) < 10


def test_forced_getrf_singular_member(handle, restore_table):
    """info and the pivots of a member with a zero column are the oracle's under folding."""
    assert rs.set_tuning_table("getrf d 200 256 1 32 64 1\n") == rs.SUCCESS
    A = uniform_general(200, 200, 3, seed=9)
    A[1][:, 57] = 0.0
    LU, ipiv, info, _ = gpu_getrf(handle, A)
    assert info[1] != 0
    check_getrf(A, LU, ipiv, info)


@pytest.mark.parametrize("nt,r,jb", VB_VARIANTS)
@pytest.mark.parametrize("fold,per_sm", [(0, 0), (1, 1)])
def test_forced_vbatched_config(handle, restore_table, nt, r, jb, fold, per_sm):
    import torch
    nmax = min(nt * r, 300)
    assert rs.set_tuning_table(f"vbatched d {nmax} {nt} {r} {jb} 64 {fold} {per_sm}\n") \
        == rs.SUCCESS
    bc = 24
    rng = np.random.default_rng(nmax + fold)
    sizes = rng.integers(8, nmax + 1, bc).astype(np.int32)
    sizes[0] = nmax
    rhs = rng.integers(1, 5, bc).astype(np.int32)
    A0 = rng.uniform(-1, 1, (bc, nmax, nmax)) + 0.1 * sizes[:, None, None] * np.eye(nmax)
    B0 = rng.uniform(-1, 1, (bc, 4, nmax))
    dA = torch.from_numpy(np.ascontiguousarray(np.transpose(A0, (0, 2, 1)))).cuda()
    dB = torch.from_numpy(B0.copy()).cuda()
    ds = torch.from_numpy(sizes).cuda()
    dr = torch.from_numpy(rhs).cuda()
    ld = torch.full((bc,), nmax, dtype=torch.int32, device="cuda")
    ipiv = torch.zeros(bc * nmax, dtype=torch.int32, device="cuda")
    info = torch.full((bc,), -9, dtype=torch.int32, device="cuda")
    ar = torch.arange(bc, device="cuda", dtype=torch.int64)
    pa = ar * (nmax * nmax * 8) + dA.data_ptr()
    pb = ar * (4 * nmax * 8) + dB.data_ptr()
    pp = ar * (nmax * 4) + ipiv.data_ptr()
    P = rs.ptr
    st = rs.call("rocsolver_dgesv_vbatched", handle, P(ds), P(dr), P(pa), P(ld), P(pp), P(pb),
                 P(ld), P(info), nmax, 4, bc)
    assert st == rs.SUCCESS
    torch.cuda.synchronize()
    assert np.all(info.cpu().numpy() == 0)
    X = dB.cpu().numpy()
    for b in range(bc):
        n, k = int(sizes[b]), int(rhs[b])
        Ab = A0[b, :n, :n]
        xb = X[b, :k, :n].T
        bb = B0[b, :k, :n].T
        res = np.abs(Ab @ xb - bb).max() / (np.abs(Ab).sum(1).max() * np.abs(xb).max())
        assert res / (n * np.finfo(np.float64).eps) < 10, (b, n)
