"""Error metrics of the reference's test clients (clients/include/norm.hpp:16-112)
and the backward errors reported for the benchmarked configurations."""
import numpy as np

EPS = {np.float64: np.finfo(np.float64).eps, np.float32: np.finfo(np.float32).eps}


def eps_of(dtype):
    return float(np.finfo(dtype).eps)


def _lange(kind, M):
    M = np.abs(np.asarray(M)).astype(np.float64)  # modulus for complex entries (zlange)
    if M.size == 0:
        return 0.0
    if kind == "F":
        return float(np.sqrt((M * M).sum()))
    if kind == "I":  # max absolute row sum
        return float(M.sum(axis=1).max())
    if kind == "O":  # max absolute column sum
        return float(M.sum(axis=0).max())
    if kind == "M":
        return float(M.max())
    raise ValueError(kind)


def norm_error(kind, ref, test):
    """||ref - test|| / ||ref|| (norm.hpp:68-90).  Returns 0 for a zero reference
    that is matched exactly."""
    wide = np.complex128 if np.iscomplexobj(ref) or np.iscomplexobj(test) else np.float64
    ref = np.asarray(ref, dtype=wide)
    test = np.asarray(test, dtype=wide)
    d = _lange(kind, ref - test)
    r = _lange(kind, ref)
    if r == 0.0:
        return 0.0 if d == 0.0 else np.inf
    return d / r


def norm_error_lower(kind, ref, test):
    return norm_error(kind, np.tril(ref), np.tril(test))


def norm_error_upper(kind, ref, test):
    return norm_error(kind, np.triu(ref), np.triu(test))


def lu_backward_error(A, LU, ipiv):
    """||P A - L U||_1 / (n ||A||_1 eps)-style numerator: returns
    ||PA - LU||_F / ||A||_F for one square member (caller divides by n*eps)."""
    n = A.shape[0]
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    PA = A.copy()
    for k in range(n):
        p = ipiv[k] - 1
        if p != k:
            PA[[k, p]] = PA[[p, k]]
    return _lange("F", PA - L @ U) / max(_lange("F", A), 1e-300)


def solve_backward_error(A, X, B):
    """||A X - B||_inf / (||A||_inf ||X||_inf + ||B||_inf), computed in long double."""
    A = np.asarray(A, dtype=np.longdouble)
    X = np.asarray(X, dtype=np.longdouble)
    B = np.asarray(B, dtype=np.longdouble)
    R = A @ X - B
    num = float(np.abs(R).sum(axis=1).max()) if R.size else 0.0
    den = float(np.abs(A).sum(axis=1).max() * np.abs(X).sum(axis=1).max()
                + np.abs(B).sum(axis=1).max())
    return num / den if den > 0 else num
