"""The bounds-checked debug build (librocsolver_b200_checked.so, -DRSB_BOUNDS_CHECK): every
element access of the factor and solve kernels is checked against the matrix dimensions and
every pivot index against 1..n; a violation is recorded, not performed (the reference's
analogue is its ROCSOLVER_VERIFY_ASSUMPTIONS build, library/src/include/lib_host_helpers.hpp:
63-80).  The normal library reports that no checks are compiled in.  The GPU test runs the
checked library in a child process (the parent has loaded the normal one) on odd sizes,
padded leading dimensions and pointer-array batches, compares with the oracle, and requires a
clean record."""
import os
import subprocess
import sys

import pytest

import rocsolver_b200 as rs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_normal_library_has_no_checks():
    import ctypes
    out = (ctypes.c_int32 * 4)()
    assert rs.call("rocsolver_b200_bounds_check", ctypes.cast(out, ctypes.c_void_p)) \
        == rs.NOT_IMPLEMENTED


def test_checked_library_exports_the_same_symbols():
    if not os.path.exists(rs.CHECKED_LIB_PATH):
        pytest.skip("bounds-checked library not built (python -m rocsolver_b200.build --checked)")

    def syms(path):
        out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                             check=True).stdout
        return {l.split()[-1] for l in out.splitlines() if l.split()[-1].startswith(("rocsolver_",
                                                                                     "rocblas_"))}
    assert syms(rs.CHECKED_LIB_PATH) == syms(rs.LIB_PATH)


CHILD = r'''
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, ROOT)
import oracle
import rocsolver_b200 as rs
from tests.refcases import to_colmajor, from_colmajor, uniform_general, spd_gram
from tests.gpu_util import ptr_array
assert rs.LIB_PATH.endswith("_checked.so"), rs.LIB_PATH
h = rs.Handle(torch.cuda.current_stream().cuda_stream)
P = rs.ptr
rec = (ctypes.c_int32 * 4)()
def check_clean(what):
    torch.cuda.synchronize()
    assert rs.call("rocsolver_b200_bounds_check", ctypes.cast(rec, ctypes.c_void_p)) == rs.SUCCESS
    assert rec[0] == 0, (what, list(rec))
for n in (1, 3, 17, 31, 32, 33, 63, 65, 100, 129, 257):
    for m in (n, n + 5):
        lda = m + 3
        A = uniform_general(m, n, 3, seed=n * 13 + m)
        dA = torch.from_numpy(to_colmajor(A, lda)).cuda()
        dP = torch.zeros(3 * min(m, n), dtype=torch.int32, device="cuda")
        dI = torch.zeros(3, dtype=torch.int32, device="cuda")
        rs.check(rs.call("rocsolver_dgetrf_strided_batched", h.value, m, n, P(dA), lda, lda * n,
                         P(dP), min(m, n), P(dI), 3), "getrf")
        check_clean(("getrf", m, n))
        oA = to_colmajor(A)
        oP, oI = np.zeros(3 * min(m, n), np.int32), np.zeros(3, np.int32)
        oracle.getrf(m, n, oA, m, m * n, oP, min(m, n), oI, 3)
        assert np.array_equal(dP.cpu().numpy(), oP) and np.array_equal(dI.cpu().numpy(), oI), (m, n)
    B = uniform_general(n, 2, 3, seed=n)
    A = uniform_general(n, n, 3, seed=n + 1)
    ldb = n + 2
    dA = torch.from_numpy(to_colmajor(A)).cuda()
    dB = torch.from_numpy(to_colmajor(B, ldb)).cuda()
    dP = torch.zeros(3 * n, dtype=torch.int32, device="cuda")
    dI = torch.zeros(3, dtype=torch.int32, device="cuda")
    aA, aB = ptr_array(dA, 3, n * n), ptr_array(dB, 3, ldb * 2)
    rs.check(rs.call("rocsolver_dgesv_batched", h.value, n, 2, P(aA), n, P(dP), n, P(aB), ldb,
                     P(dI), 3), "gesv_batched")
    for op in (rs.OP_N, rs.OP_T):
        rs.check(rs.call("rocsolver_dgetrs_strided_batched", h.value, op, n, 2, P(dA), n, n * n,
                         P(dP), n, P(dB), ldb, ldb * 2, 3), "getrs")
    check_clean(("gesv/getrs", n))
    S = spd_gram(n, 2, seed=n)
    dS = torch.from_numpy(to_colmajor(S, n + 1)).cuda()
    dJ = torch.zeros(2, dtype=torch.int32, device="cuda")
    rs.check(rs.call("rocsolver_dpotrf_strided_batched", h.value, rs.FILL_LOWER, n, P(dS), n + 1,
                     (n + 1) * n, P(dJ), 2), "potrf")
    check_clean(("potrf", n))
    # complex: zgetrf (rectangular, then square) with a padded leading dimension, zgetrs
    # N / T / C on the square factors, zposv upper
    Z = (uniform_general(n + 2, n, 2, seed=n) + 1j * uniform_general(n + 2, n, 2, seed=n + 7))
    dZ = torch.from_numpy(to_colmajor(Z, n + 4)).cuda()
    dP = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    dI = torch.zeros(2, dtype=torch.int32, device="cuda")
    rs.check(rs.call("rocsolver_zgetrf_strided_batched", h.value, n + 2, n, P(dZ), n + 4,
                     (n + 4) * n, P(dP), n, P(dI), 2), "zgetrf")
    dZ = torch.from_numpy(to_colmajor(Z[:, :n, :].copy(), n + 4)).cuda()
    rs.check(rs.call("rocsolver_zgetrf_strided_batched", h.value, n, n, P(dZ), n + 4,
                     (n + 4) * n, P(dP), n, P(dI), 2), "zgetrf")
    dZB = torch.from_numpy(to_colmajor(Z[:, :n, :2].copy(), n + 1)).cuda()
    for op in (rs.OP_N, rs.OP_T, rs.OP_C):
        rs.check(rs.call("rocsolver_zgetrs_strided_batched", h.value, op, n, 2, P(dZ), n + 4,
                         (n + 4) * n, P(dP), n, P(dZB), n + 1, (n + 1) * 2, 2), "zgetrs")
    H = spd_gram(n, 2, seed=n).astype(np.complex128)
    dH = torch.from_numpy(to_colmajor(H, n + 1)).cuda()
    rs.check(rs.call("rocsolver_zposv_strided_batched", h.value, rs.FILL_UPPER, n, 2, P(dH), n + 1,
                     (n + 1) * n, P(dZB), n + 1, (n + 1) * 2, P(dI), 2), "zposv")
    check_clean(("complex", n))
h.close()
print("bounds clean")
'''


@pytest.mark.gpu
def test_checked_build_runs_clean_on_odd_sizes():
    if not os.path.exists(rs.CHECKED_LIB_PATH):
        pytest.skip("bounds-checked library not built (python -m rocsolver_b200.build --checked)")
    env = dict(os.environ, ROCSOLVER_B200_LIB=rs.CHECKED_LIB_PATH)
    code = "ROOT = " + repr(ROOT) + "\n" + CHILD
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "bounds clean" in r.stdout
