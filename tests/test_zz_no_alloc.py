"""GPU test of rocsolver_dgesv_vbatched_noalloc, the variable-size solve for callers that
may not allocate device memory (it keeps its work list in a fixed array inside the library
instead of the handle's cudaMalloc'd workspace).  Through the C ABI, two calls in a row
must reproduce the allocating rocsolver_dgesv_vbatched on the same inputs (pivots and info
exactly, solutions to 1e-12 relative), and an over-limit batch must be rejected.

This file is collected last on purpose, so a run that stops at the first failure has run
every other test before it; it also passes on its own in a fresh process."""
import numpy as np
import pytest

import rocsolver_b200 as rs

pytestmark = pytest.mark.gpu

MAX_BATCH = 1 << 20


def make_batch(torch, seed, ns, nrs):
    """Members packed in one device buffer; returns device tensors and pointer arrays."""
    rng = np.random.default_rng(seed)
    nmax, rmax = max(ns), max(nrs)
    bc = len(ns)
    A = np.zeros((bc, nmax * nmax))
    B = np.zeros((bc, nmax * rmax))
    for i, (n, r) in enumerate(zip(ns, nrs)):
        M = rng.uniform(-1, 1, (n, n)) + 0.1 * n * np.eye(n)
        A[i, : n * n] = M.T.reshape(-1)          # column-major, lda = n
        B[i, : n * r] = rng.uniform(-1, 1, (r, n)).reshape(-1)
    dA = torch.from_numpy(A).cuda()
    dB = torch.from_numpy(B).cuda()
    dP = torch.zeros(bc, nmax, dtype=torch.int32, device="cuda")
    dI = torch.full((bc,), -7, dtype=torch.int32, device="cuda")
    rows = torch.arange(bc, device="cuda", dtype=torch.int64)
    pA = rows * (nmax * nmax * 8) + dA.data_ptr()
    pB = rows * (nmax * rmax * 8) + dB.data_ptr()
    pP = rows * (nmax * 4) + dP.data_ptr()
    dn = torch.tensor(ns, dtype=torch.int32, device="cuda")
    dr = torch.tensor(nrs, dtype=torch.int32, device="cuda")
    return dict(A=dA, B=dB, P=dP, I=dI, pA=pA, pB=pB, pP=pP, n=dn, r=dr, bc=bc, nmax=nmax,
                rmax=rmax)


def solve(name, handle, d):
    return rs.call(name, handle, rs.ptr(d["n"]), rs.ptr(d["r"]), rs.ptr(d["pA"]), rs.ptr(d["n"]),
                   rs.ptr(d["pP"]), rs.ptr(d["pB"]), rs.ptr(d["n"]), rs.ptr(d["I"]), d["nmax"],
                   d["rmax"], d["bc"])


def test_noalloc_matches_allocating_vbatched_twice():
    import torch
    h = rs.Handle(torch.cuda.current_stream().cuda_stream)
    try:
        rng = np.random.default_rng(11)
        ns = [int(x) for x in rng.integers(1, 140, 300)] + [1, 32, 33, 200]
        nrs = [int(x) for x in rng.integers(1, 9, len(ns))]
        ref = make_batch(torch, 5, ns, nrs)
        A0, B0 = ref["A"].clone(), ref["B"].clone()
        assert solve("rocsolver_dgesv_vbatched", h.value, ref) == rs.SUCCESS
        torch.cuda.synchronize()
        for call in range(2):  # two calls in a row through the shared scratch array
            d = make_batch(torch, 5, ns, nrs)
            assert torch.equal(d["A"], A0) and torch.equal(d["B"], B0)
            st = solve("rocsolver_dgesv_vbatched_noalloc", h.value, d)
            assert st == rs.SUCCESS, rs.STATUS_NAMES[st]
            torch.cuda.synchronize()
            assert torch.equal(d["I"], ref["I"]), call
            assert not d["I"].any()
            assert torch.equal(d["P"], ref["P"]), call
            err = ((d["B"] - ref["B"]).abs().max() / ref["B"].abs().max()).item()
            assert err <= 1e-12, (call, err)
            lu_err = ((d["A"] - ref["A"]).abs().max() / ref["A"].abs().max()).item()
            assert lu_err <= 1e-12, (call, lu_err)
    finally:
        h.close()


def test_noalloc_rejects_batches_over_the_limit():
    import torch
    h = rs.Handle(torch.cuda.current_stream().cuda_stream)
    try:
        fake = rs.ptr(torch.zeros(1, device="cuda"))
        st = rs.call("rocsolver_dgesv_vbatched_noalloc", h.value, fake, fake, fake, fake, fake,
                     fake, fake, fake, 8, 1, MAX_BATCH + 1)
        assert st == rs.INVALID_SIZE
        st = rs.call("rocsolver_dgesv_vbatched_noalloc", None, fake, fake, fake, fake, fake,
                     fake, fake, fake, 8, 1, 4)
        assert st == rs.INVALID_HANDLE
    finally:
        h.close()
