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


def test_noalloc_matches_oracle_near_max_n():
    """The no-allocation solve against the oracle directly (ipiv and info exact, backward
    error < 10 n eps), with members up to max_n = 320 and one of order max_n itself."""
    import oracle
    import torch
    from tests.norms import solve_backward_error
    h = rs.Handle(torch.cuda.current_stream().cuda_stream)
    try:
        rng = np.random.default_rng(23)
        ns = [int(x) for x in rng.integers(1, 320, 40)] + [320, 33, 1]
        nrs = [int(x) for x in rng.integers(1, 9, len(ns))]
        d = make_batch(torch, 29, ns, nrs)
        A0 = d["A"].cpu().numpy().copy()
        B0 = d["B"].cpu().numpy().copy()
        st = solve("rocsolver_dgesv_vbatched_noalloc", h.value, d)
        assert st == rs.SUCCESS, rs.STATUS_NAMES[st]
        torch.cuda.synchronize()
        P, I, X = d["P"].cpu().numpy(), d["I"].cpu().numpy(), d["B"].cpu().numpy()
        eps = np.finfo(np.float64).eps
        for i, (n, r) in enumerate(zip(ns, nrs)):
            oA = A0[i, : n * n].copy()
            oB = B0[i, : n * r].copy()
            oP, oI = np.zeros(n, np.int32), np.zeros(1, np.int32)
            oracle.gesv(n, r, oA, n, n * n, oP, n, oB, n, n * r, oI, 1)
            assert I[i] == oI[0]
            np.testing.assert_array_equal(P[i, :n], oP, err_msg=f"member {i} n={n}")
            M = A0[i, : n * n].reshape(n, n).T
            x = X[i, : n * r].reshape(r, n).T
            b = B0[i, : n * r].reshape(r, n).T
            assert solve_backward_error(M, x, b) < 10 * n * eps, (i, n)
    finally:
        h.close()


def test_noalloc_edge_members_match_allocating_vbatched():
    """Members the plan kernel must reject or that fail, and a batch of only small members
    (no member for the CTA path): info, ipiv and B exactly those of the allocating
    rocsolver_dgesv_vbatched.  Batch 1: n > max_n, lda < n, nrhs > max_nrhs (info -1,
    member untouched), a singular member (info > 0, B unchanged) and valid members."""
    import torch
    h = rs.Handle(torch.cuda.current_stream().cuda_stream)
    try:
        def run(name, ns, nrs, lds, max_n, max_nrhs, singular=()):
            d = make_batch(torch, 31, [max(x, 1) for x in ns], nrs)
            for i in singular:  # a zero column makes the member exactly singular
                n = ns[i]
                d["A"][i, (n // 2) * n: (n // 2) * n + n] = 0.0
            d["n"] = torch.tensor(ns, dtype=torch.int32, device="cuda")
            d["ld"] = torch.tensor(lds, dtype=torch.int32, device="cuda")
            d["nmax"], d["rmax"] = max_n, max_nrhs
            st = rs.call(name, h.value, rs.ptr(d["n"]), rs.ptr(d["r"]), rs.ptr(d["pA"]),
                         rs.ptr(d["ld"]), rs.ptr(d["pP"]), rs.ptr(d["pB"]), rs.ptr(d["ld"]),
                         rs.ptr(d["I"]), max_n, max_nrhs, d["bc"])
            assert st == rs.SUCCESS, rs.STATUS_NAMES[st]
            torch.cuda.synchronize()
            return d

        ns = [40, 90, 50, 60, 30, 70]
        nrs = [2, 1, 3, 20, 4, 2]
        lds = [40, 90, 45, 60, 30, 70]   # member 2: lda 45 < n 50
        ns_call = [40, 90, 50, 60, 30, 70]
        ns_call[1] = 90                   # member 1: n 90 > max_n 80
        for i in range(2):
            ref = run("rocsolver_dgesv_vbatched", ns_call, nrs, lds, 80, 16, singular=(4,))
            got = run("rocsolver_dgesv_vbatched_noalloc", ns_call, nrs, lds, 80, 16,
                      singular=(4,))
            info = got["I"].cpu().numpy()
            assert info[1] == -1 and info[2] == -1 and info[3] == -1, info
            assert info[4] > 0 and info[0] == 0 and info[5] == 0, info
            for k in ("I", "P", "B", "A"):
                assert torch.equal(got[k], ref[k]), (i, k)
        small = [int(x) for x in np.random.default_rng(3).integers(1, 33, 70)]
        snr = [1 + (x % 5) for x in small]
        for i in range(2):
            ref = run("rocsolver_dgesv_vbatched", small, snr, small, 32, 5)
            got = run("rocsolver_dgesv_vbatched_noalloc", small, snr, small, 32, 5)
            assert not got["I"].any()
            for k in ("I", "P", "B", "A"):
                assert torch.equal(got[k], ref[k]), (i, k)
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
