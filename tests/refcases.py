"""Input generators shared by the tests and the golden-fixture script.

Matrices are returned as numpy arrays of shape (batch, rows, cols), element
(i, j) of member b at [b, i, j].  ``to_colmajor`` packs them into the flat
column-major (lda, stride) layout of the reference API.

Reference-style generators reproduce rocSOLVER's own test inputs exactly
(clients/include/testing_*.hpp initData functions); see oracle/refgen.cpp for
the integer stream.
"""
import numpy as np


def _refstream(count, cplx=False):
    """count values of the reference's integer stream; complex values take two draws each,
    real part first (clients/rocblascommon/rocblas_random.hpp random_generator for
    rocblas_float_complex / rocblas_double_complex)."""
    import oracle
    if not cplx:
        return oracle.refgen(count)
    v = oracle.refgen(2 * count)
    return v[0::2] + 1j * v[1::2]


def _member_view(flat, bc, ld, ncols):
    # flat buffer filled in memory order -> (bc, ld, ncols) with column-major members
    return flat.reshape(bc, ncols, ld).transpose(0, 2, 1).copy()


def ref_getrf_input(m, n, lda, bc, singular, cplx=False):
    """clients/include/testing_getf2_getrf.hpp:128-180 (the +400 / -4 act on the real part
    of a complex element)."""
    A = _member_view(_refstream(bc * lda * n, cplx), bc, lda, n)
    for b in range(bc):
        for i in range(m):
            for j in range(n):
                A[b, i, j] += 400.0 if i == j else -4.0
        A[b, :m, :] = A[b, :m, :][::-1, :].copy()
        if singular and (b == bc // 4 or b == bc // 2 or b == bc - 1):
            for j0 in (n // 4 + b, n // 2 + b, n - 1 + b):
                A[b, :m, j0 % n] = 0.0
    return A[:, :m, :].copy()


def ref_getrs_input(n, nrhs, bc, cplx=False):
    """clients/include/testing_getrs.hpp:125-160 (A before its host getrf, and B)."""
    A = _member_view(_refstream(bc * n * n, cplx), bc, n, n)
    B = _member_view(_refstream(bc * n * nrhs, cplx), bc, n, nrhs)
    idx = np.arange(n)
    for b in range(bc):
        A[b] -= 4.0
        A[b, idx, idx] += 404.0
    return A, B


def ref_gesv_input(n, nrhs, bc, singular, cplx=False):
    """clients/include/testing_gesv.hpp:138-180."""
    A, B = ref_getrs_input(n, nrhs, bc, cplx)
    if singular:
        for b in range(bc):
            if b == bc // 4 or b == bc // 2 or b == bc - 1:
                for j0 in (n // 4 + b, n // 2 + b, n - 1 + b):
                    A[b, :, j0 % n] = 0.0
    return A, B


def ref_potrf_input(n, bc, singular, cplx=False):
    """clients/include/testing_potf2_potrf.hpp:103-140 (non-symmetric; only the
    referenced triangle matters; the diagonal becomes a * conj(a) * 400, real)."""
    A = _member_view(_refstream(bc * n * n, cplx), bc, n, n)
    idx = np.arange(n)
    for b in range(bc):
        A[b, idx, idx] = A[b, idx, idx] * np.conj(A[b, idx, idx]) * 400.0
        if singular and (b == bc // 4 or b == bc // 2 or b == bc - 1):
            for i0 in (n // 4 + b, n // 2 + b, n - 1 + b):
                A[b, i0 % n, i0 % n] = 0.0
    return A


def ref_getri_matrix(n, lda, bc, cplx=False):
    """clients/include/testing_getri.hpp:102-150 before its host getrf: integers 1..10 scaled
    to v/10 + 10 on the diagonal and (v - 4)/10 off it, rows reversed (complex: the shifts
    act on the real part)."""
    A = _member_view(_refstream(bc * lda * n, cplx), bc, lda, n)[:, :n, :].copy()
    idx = np.arange(n)
    for b in range(bc):
        M = (A[b] - 4.0) / 10.0
        M[idx, idx] = A[b][idx, idx] / 10.0 + 10.0
        A[b] = M[::-1, :]
    return A


def ref_getri_singular(b, bc, n):
    """Diagonal positions of U zeroed in the reference's singular getri members
    (testing_getri.hpp:150-166), or () for a regular member."""
    if b == bc // 4 or b == bc // 2 or b == bc - 1:
        return tuple(sorted({(n // 4 + b) % n, (n // 2 + b) % n, (n - 1 + b) % n}))
    return ()


def uniform_general(m, n, bc, seed, lo=-1.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, size=(bc, m, n))


def uniform_complex(m, n, bc, seed):
    """Real and imaginary parts independent uniform[-1, 1]."""
    r = np.random.default_rng(seed).uniform(-1.0, 1.0, size=(2, bc, m, n))
    return r[0] + 1j * r[1]


def hpd_gram(n, bc, seed):
    """Hermitian positive definite A = G G^H + n I with G complex Gaussian."""
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((bc, n, n)) + 1j * rng.standard_normal((bc, n, n))
    return G @ np.conj(G.transpose(0, 2, 1)) + n * np.eye(n)[None]


def cond_graded(n, bc, seed, lo=1.0, hi=6.0):
    """A = U diag(s) V^T with U, V orthogonal (QR of Gaussians) and s log-spaced from 1 to
    1/kappa, log10(kappa) ~ U[lo, hi] per member: the mixed-precision configuration's input
    distribution, generated on the host with numpy."""
    rng = np.random.default_rng(seed)
    out = np.empty((bc, n, n))
    t = np.linspace(0.0, 1.0, n)
    for b in range(bc):
        U, _ = np.linalg.qr(rng.standard_normal((n, n)))
        V, _ = np.linalg.qr(rng.standard_normal((n, n)))
        lk = lo + (hi - lo) * rng.uniform()
        out[b] = (U * 10.0 ** (-lk * t)[None, :]) @ V.T
    return out


def projections(M, seed=7, k=4):
    """(M @ V, W^T @ M) for seeded N(0,1) V (n x k) and W (m x k): a compact fingerprint of
    a large factor, so that golden fixtures of big members stay small."""
    rng = np.random.default_rng(seed)
    m, n = M.shape
    V = rng.standard_normal((n, k))
    W = rng.standard_normal((m, k))
    return M @ V, W.T @ M, V, W


def spd_gram(n, bc, seed):
    """A = G G^T + n I with G ~ N(0,1) (the Cholesky configuration's inputs)."""
    G = np.random.default_rng(seed).standard_normal((bc, n, n))
    return G @ G.transpose(0, 2, 1) + n * np.eye(n)[None]


def to_colmajor(A, ld=None, stride=None, dtype=None):
    """(bc, m, n) -> flat column-major buffer with leading dimension ld and
    member stride (elements); padding is filled with NaN so stray reads and
    writes show up."""
    bc, m, n = A.shape
    ld = m if ld is None else ld
    stride = ld * n if stride is None else stride
    dtype = A.dtype if dtype is None else dtype
    flat = np.full(max(stride * bc, 1), np.nan, dtype=dtype)
    for b in range(bc):
        blk = np.full((n, ld), np.nan, dtype=dtype)
        blk[:, :m] = A[b].T
        flat[b * stride: b * stride + ld * n] = blk.reshape(-1)
    return flat


def from_colmajor(flat, bc, m, n, ld, stride):
    out = np.empty((bc, m, n), dtype=flat.dtype)
    for b in range(bc):
        out[b] = flat[b * stride: b * stride + ld * n].reshape(n, ld).T[:m, :]
    return out
