"""GPU tests of the variable-size batched path (rocsolver_{s,d}{gesv,getrf,getrs}_vbatched):
against the oracle member by member (ipiv/info exact, backward error), against per-size
separate launches of the fixed-size entry points, invalid members, and CUDA-graph capture
of the whole call."""
import numpy as np
import pytest

import oracle
import rocsolver_b200 as rs
from tests.gpu_util import GpuHandle, dev, host, prefix, ptr
from tests.norms import eps_of, solve_backward_error

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    h = GpuHandle()
    yield h.value
    h.close()


class VBatch:
    """Members packed back to back in one device buffer; pointer arrays into it."""

    def __init__(self, ns, nrhss, dtype, seed, pad=0):
        import torch
        rng = np.random.default_rng(seed)
        self.ns, self.nrhss = list(ns), list(nrhss)
        self.dtype = dtype
        self.As, self.Bs = [], []
        offA, offB, offP = [], [], []
        ta = tb = tp = 0
        for n, r in zip(ns, nrhss):
            A = rng.uniform(-1, 1, (n, n)) + 0.1 * n * np.eye(n)
            B = rng.uniform(-1, 1, (n, r))
            self.As.append(A.astype(dtype))
            self.Bs.append(B.astype(dtype))
            lda = n + pad
            offA.append(ta)
            ta += lda * n + 3
            offB.append(tb)
            tb += lda * r + 1
            offP.append(tp)
            tp += n + 1
        self.ld = [n + pad for n in ns]
        flatA = np.full(ta, np.nan, dtype)
        flatB = np.full(tb, np.nan, dtype)
        for i, (A, B) in enumerate(zip(self.As, self.Bs)):
            n, r, ld = self.ns[i], self.nrhss[i], self.ld[i]
            blk = np.full((n, ld), np.nan, dtype)
            blk[:, :n] = A.T
            flatA[offA[i]: offA[i] + ld * n] = blk.reshape(-1)
            blk = np.full((r, ld), np.nan, dtype)
            blk[:, :n] = B.T
            flatB[offB[i]: offB[i] + ld * r] = blk.reshape(-1)
        self.dA, self.dB = dev(flatA), dev(flatB)
        self.dP = dev(np.zeros(max(tp, 1), np.int32))
        es = np.dtype(dtype).itemsize
        self.pA = torch.tensor([self.dA.data_ptr() + o * es for o in offA], dtype=torch.int64,
                               device="cuda")
        self.pB = torch.tensor([self.dB.data_ptr() + o * es for o in offB], dtype=torch.int64,
                               device="cuda")
        self.pP = torch.tensor([self.dP.data_ptr() + o * 4 for o in offP], dtype=torch.int64,
                               device="cuda")
        self.dn = dev(np.array(ns, np.int32))
        self.dr = dev(np.array(nrhss, np.int32))
        self.dld = dev(np.array(self.ld, np.int32))
        self.dI = dev(np.full(len(ns), -5, np.int32))
        self.offA, self.offB, self.offP = offA, offB, offP

    def results(self):
        fa, fb, fp, info = host(self.dA), host(self.dB), host(self.dP), host(self.dI)
        LU, X, P = [], [], []
        for i, (n, r, ld) in enumerate(zip(self.ns, self.nrhss, self.ld)):
            LU.append(fa[self.offA[i]: self.offA[i] + ld * n].reshape(n, ld).T[:n])
            X.append(fb[self.offB[i]: self.offB[i] + ld * r].reshape(r, ld).T[:n])
            P.append(fp[self.offP[i]: self.offP[i] + n])
        return LU, X, P, info


def run_gesv_vb(handle, vb, max_n, max_nrhs):
    p = prefix(vb.dtype)
    return rs.call(f"rocsolver_{p}gesv_vbatched", handle, ptr(vb.dn), ptr(vb.dr), ptr(vb.pA),
                   ptr(vb.dld), ptr(vb.pP), ptr(vb.pB), ptr(vb.dld), ptr(vb.dI), max_n, max_nrhs,
                   len(vb.ns))


def check_against_oracle(vb, LU, X, P, info):
    eps = eps_of(vb.dtype)
    for i, (A, B) in enumerate(zip(vb.As, vb.Bs)):
        n, r = A.shape[0], B.shape[1]
        oA = A.T.copy().reshape(-1)
        oB = B.T.copy().reshape(-1)
        oP, oI = np.zeros(n, np.int32), np.zeros(1, np.int32)
        oracle.gesv(n, r, oA, n, n * n, oP, n, oB, n, n * r, oI, 1)
        assert info[i] == oI[0], i
        np.testing.assert_array_equal(P[i], oP, err_msg=f"member {i} n={n}")
        be = solve_backward_error(A.astype(np.float64), X[i].astype(np.float64),
                                  B.astype(np.float64))
        assert be < 10 * n * eps, (i, n, be)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_gesv_vbatched_mixed_sizes(handle, dtype):
    rng = np.random.default_rng(1)
    ns = list(rng.integers(1, 90, 150)) + [200, 257, 300, 31, 32, 33, 1, 2]
    nr = list(rng.integers(1, 17, len(ns)))
    vb = VBatch(ns, nr, dtype, seed=2, pad=2)
    assert run_gesv_vb(handle, vb, 300, 16) == rs.SUCCESS
    check_against_oracle(vb, *vb.results())


def test_gesv_vbatched_matches_per_size_launches(handle):
    """Same members solved through per-size separate gesv_batched launches give identical
    ipiv/info and solutions within rounding."""
    rng = np.random.default_rng(3)
    ns = list(rng.choice([8, 40, 64, 130], 60))
    nr = [4] * len(ns)
    vb = VBatch(ns, nr, np.float64, seed=4)
    assert run_gesv_vb(handle, vb, 130, 4) == rs.SUCCESS
    LU, X, P, info = vb.results()
    for n in sorted(set(ns)):
        idx = [i for i, v in enumerate(ns) if v == n]
        A = np.stack([vb.As[i] for i in idx])
        B = np.stack([vb.Bs[i] for i in idx])
        from tests.refcases import from_colmajor, to_colmajor
        dA, dB = dev(to_colmajor(A)), dev(to_colmajor(B))
        dP = dev(np.zeros(len(idx) * n, np.int32))
        dI = dev(np.zeros(len(idx), np.int32))
        rs.check(rs.call("rocsolver_dgesv_strided_batched", handle, n, 4, ptr(dA), n, n * n,
                         ptr(dP), n, ptr(dB), n, n * 4, ptr(dI), len(idx)), "gesv")
        Xs = from_colmajor(host(dB), len(idx), n, 4, n, n * 4)
        Ps = host(dP).reshape(len(idx), n)
        for k, i in enumerate(idx):
            np.testing.assert_array_equal(P[i], Ps[k])
            assert np.abs(X[i] - Xs[k]).max() <= 1e-12 * max(1.0, np.abs(Xs[k]).max())


def test_getrf_getrs_vbatched_pair(handle):
    rng = np.random.default_rng(5)
    ns = list(rng.integers(1, 120, 40))
    nr = list(rng.integers(1, 6, 40))
    vb = VBatch(ns, nr, np.float64, seed=6)
    rs.check(rs.call("rocsolver_dgetrf_vbatched", handle, ptr(vb.dn), ptr(vb.pA), ptr(vb.dld),
                     ptr(vb.pP), ptr(vb.dI), 119, len(ns)), "getrf_vbatched")
    rs.check(rs.call("rocsolver_dgetrs_vbatched", handle, ptr(vb.dn), ptr(vb.dr), ptr(vb.pA),
                     ptr(vb.dld), ptr(vb.pP), ptr(vb.pB), ptr(vb.dld), 119, 5, len(ns)),
             "getrs_vbatched")
    check_against_oracle(vb, *vb.results())


def test_vbatched_invalid_member(handle):
    vb = VBatch([10, 20, 30], [1, 1, 1], np.float64, seed=7)
    # member 1 claims n = 50 > max_n = 40 -> info = -1, untouched
    import torch
    vb.dn.copy_(torch.tensor([10, 50, 30], dtype=torch.int32))
    before = host(vb.dA).copy()
    assert run_gesv_vb(handle, vb, 40, 1) == rs.SUCCESS
    info = host(vb.dI)
    assert info[1] == -1 and info[0] == 0 and info[2] == 0
    after = host(vb.dA)
    s, e = vb.offA[1], vb.offA[1] + 20 * 20
    np.testing.assert_array_equal(after[s:e], before[s:e])


def test_gesv_vbatched_cuda_graph(handle):
    """The whole variable-size call captured in a CUDA graph and replayed: same results
    as the eager call."""
    import torch
    rng = np.random.default_rng(8)
    ns = list(rng.integers(8, 200, 64))
    nr = list(rng.integers(1, 17, 64))
    vb = VBatch(ns, nr, np.float64, seed=9)
    A0, B0 = vb.dA.clone(), vb.dB.clone()
    s = torch.cuda.Stream()
    h = rs.Handle(s.cuda_stream)
    try:
        with torch.cuda.stream(s):
            assert run_gesv_vb(h.value, vb, 199, 16) == rs.SUCCESS  # eager (sizes workspace)
        torch.cuda.synchronize()
        eager = [x.copy() for x in vb.results()[1]]
        vb.dA.copy_(A0)
        vb.dB.copy_(B0)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            st = run_gesv_vb(h.value, vb, 199, 16)
        assert st == rs.SUCCESS
        for _ in range(2):
            vb.dA.copy_(A0)
            vb.dB.copy_(B0)
            g.replay()
            torch.cuda.synchronize()
            LU, X, P, info = vb.results()
            assert not info.any()
            for a, b in zip(X, eager):
                np.testing.assert_array_equal(a, b)
        del g
    finally:
        h.close()
