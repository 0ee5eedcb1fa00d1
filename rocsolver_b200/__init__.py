"""rocsolver_b200 -- B200 (sm_100a) implementation of rocSOLVER's batched dense LU /
Cholesky factor-and-solve path behind the reference's C ABI.

The product is the shared library ``librocsolver_b200.so`` (C ABI declared in
include/rocsolver.h).  This module is the Python-side mirror of that interface: it loads
the library with ctypes, declares every exported entry point with the reference's
argument order, and offers thin helpers that pass torch CUDA tensors by device
pointer.  There is no fallback: if the library is missing, importing ``lib()`` raises.

Reference interface mirrored: library/include/rocsolver/rocsolver-functions.h
(getrf :5139-5349, getrs :8562-8796, gesv :8872-9108, getri :9173-9547, potrf :10188-10356,
potrs :10426-10642, posv :10718-10944, getri_outofplace :21380-21834) and
library/src/lapack/roclapack_gesv_outofplace.cpp:106-135 (gesv_outofplace).
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; $ROCSOLVER_B200_LIB names another build of the same library instead
# (e.g. the bounds-checked librocsolver_b200_checked.so)
LIB_PATH = os.environ.get("ROCSOLVER_B200_LIB") or os.path.join(_HERE, "librocsolver_b200.so")
CHECKED_LIB_PATH = os.path.join(_HERE, "librocsolver_b200_checked.so")

# rocblas_status
SUCCESS, INVALID_HANDLE, NOT_IMPLEMENTED, INVALID_POINTER, INVALID_SIZE, MEMORY_ERROR, \
    INTERNAL_ERROR, PERF_DEGRADED, SIZE_QUERY_MISMATCH, SIZE_INCREASED, SIZE_UNCHANGED, \
    INVALID_VALUE, CONTINUE, CHECK_NUMERICS_FAIL = range(14)
STATUS_NAMES = ["success", "invalid_handle", "not_implemented", "invalid_pointer",
                "invalid_size", "memory_error", "internal_error", "perf_degraded",
                "size_query_mismatch", "size_increased", "size_unchanged", "invalid_value",
                "continue", "check_numerics_fail"]
# rocblas_operation / rocblas_fill
OP_N, OP_T, OP_C = 111, 112, 113
FILL_UPPER, FILL_LOWER, FILL_FULL = 121, 122, 123

_c = ctypes
H = _c.c_void_p      # rocblas_handle
I = _c.c_int32       # rocblas_int
S = _c.c_int64       # rocblas_stride
P = _c.c_void_p      # device pointer
E = _c.c_int         # enum

# argument signatures (after the handle) per entry-point family
_SIG = {
    "getrf": [I, I, P, I, P, P],
    "getrf_batched": [I, I, P, I, P, S, P, I],
    "getrf_strided_batched": [I, I, P, I, S, P, S, P, I],
    "getrf_npvt": [I, I, P, I, P],
    "getrf_npvt_batched": [I, I, P, I, P, I],
    "getrf_npvt_strided_batched": [I, I, P, I, S, P, I],
    "getrs": [E, I, I, P, I, P, P, I],
    "getrs_batched": [E, I, I, P, I, P, S, P, I, I],
    "getrs_strided_batched": [E, I, I, P, I, S, P, S, P, I, S, I],
    "gesv": [I, I, P, I, P, P, I, P],
    "gesv_batched": [I, I, P, I, P, S, P, I, P, I],
    "gesv_strided_batched": [I, I, P, I, S, P, S, P, I, S, P, I],
    "potrf": [E, I, P, I, P],
    "potrf_batched": [E, I, P, I, P, I],
    "potrf_strided_batched": [E, I, P, I, S, P, I],
    "potrs": [E, I, I, P, I, P, I],
    "potrs_batched": [E, I, I, P, I, P, I, I],
    "potrs_strided_batched": [E, I, I, P, I, S, P, I, S, I],
    "posv": [E, I, I, P, I, P, I, P],
    "posv_batched": [E, I, I, P, I, P, I, P, I],
    "posv_strided_batched": [E, I, I, P, I, S, P, I, S, P, I],
    "getri": [I, P, I, P, P],
    "getri_batched": [I, P, I, P, S, P, I],
    "getri_strided_batched": [I, P, I, S, P, S, P, I],
    "getri_npvt": [I, P, I, P],
    "getri_npvt_batched": [I, P, I, P, I],
    "getri_npvt_strided_batched": [I, P, I, S, P, I],
    "getri_outofplace": [I, P, I, P, P, I, P],
    "getri_outofplace_batched": [I, P, I, P, S, P, I, P, I],
    "getri_outofplace_strided_batched": [I, P, I, S, P, S, P, I, S, P, I],
    "getri_npvt_outofplace": [I, P, I, P, I, P],
    "getri_npvt_outofplace_batched": [I, P, I, P, I, P, I],
    "getri_npvt_outofplace_strided_batched": [I, P, I, S, P, I, S, P, I],
    "gesv_outofplace": [I, I, P, I, P, P, I, P, I, P],
}

# families the complex precisions (c, z) export: all of them
_COMPLEX_FAMILIES = list(_SIG)

# entry points with no counterpart in the reference (declared in include/rocsolver.h)
_EXTRA = {
    "rocsolver_dsgesv_strided_batched": (_c.c_int, [H, I, I, P, I, S, P, S, P, I, S, P, I, S, P,
                                                    P, I]),
}
for _p in "sd":
    _EXTRA[f"rocsolver_{_p}getrs_adjoint_strided_batched"] = (
        _c.c_int, [H, I, I, P, I, S, P, S, P, I, S, P, I, S, P, I, S, P, I, S, I])
    _EXTRA[f"rocsolver_{_p}potrs_adjoint_strided_batched"] = (
        _c.c_int, [H, E, I, I, P, I, S, P, I, S, P, I, S, P, I, S, P, I, S, I])
    _EXTRA[f"rocsolver_{_p}getrf_vbatched"] = (_c.c_int, [H, P, P, P, P, P, I, I])
    _EXTRA[f"rocsolver_{_p}getrs_vbatched"] = (_c.c_int, [H, P, P, P, P, P, P, P, I, I, I])
    _EXTRA[f"rocsolver_{_p}gesv_vbatched"] = (_c.c_int, [H, P, P, P, P, P, P, P, P, I, I, I])
_EXTRA["rocsolver_sgetrf_tf32_strided_batched"] = (_c.c_int, [H, I, I, P, I, S, P, S, P, I])
_EXTRA["rocsolver_dgesv_vbatched_noalloc"] = (_c.c_int, [H, P, P, P, P, P, P, P, P, I, I, I])
_EXTRA["rocsolver_b200_tuning_set"] = (_c.c_int, [_c.c_char_p])
_EXTRA["rocsolver_b200_tuning_load"] = (_c.c_int, [_c.c_char_p])
_EXTRA["rocsolver_b200_tuning_get"] = (_c.c_size_t, [_c.c_char_p, _c.c_size_t])
_EXTRA["rocsolver_b200_bounds_check"] = (_c.c_int, [_c.c_void_p])

_HANDLE_FUNCS = {
    "rocblas_create_handle": (_c.c_int, [_c.POINTER(H)]),
    "rocblas_destroy_handle": (_c.c_int, [H]),
    "rocblas_set_stream": (_c.c_int, [H, _c.c_void_p]),
    "rocblas_get_stream": (_c.c_int, [H, _c.POINTER(_c.c_void_p)]),
    "rocblas_start_device_memory_size_query": (_c.c_int, [H]),
    "rocblas_stop_device_memory_size_query": (_c.c_int, [H, _c.POINTER(_c.c_size_t)]),
    "rocblas_is_device_memory_size_query": (_c.c_int, [H]),
    "rocblas_is_managing_device_memory": (_c.c_int, [H]),
    "rocblas_get_device_memory_size": (_c.c_int, [H, _c.POINTER(_c.c_size_t)]),
    "rocblas_set_device_memory_size": (_c.c_int, [H, _c.c_size_t]),
    "rocblas_set_workspace": (_c.c_int, [H, _c.c_void_p, _c.c_size_t]),
    "rocsolver_get_version_string": (_c.c_int, [_c.c_char_p, _c.c_size_t]),
    "rocsolver_get_version_string_size": (_c.c_int, [_c.POINTER(_c.c_size_t)]),
    "rocsolver_log_begin": (_c.c_int, []),
    "rocsolver_log_end": (_c.c_int, []),
    "rocsolver_log_set_layer_mode": (_c.c_int, [_c.c_uint32]),
    "rocsolver_log_set_max_levels": (_c.c_int, [I]),
    "rocsolver_log_restore_defaults": (_c.c_int, []),
    "rocsolver_log_write_profile": (_c.c_int, []),
    "rocsolver_log_flush_profile": (_c.c_int, []),
}

_lib = None


def entry_points():
    """Every exported entry point name (reference ones first, then the handle shim and
    the new ones)."""
    names = [f"rocsolver_{p}{f}" for p in "sd" for f in _SIG]
    names += [f"rocsolver_{p}{f}" for p in "cz" for f in _COMPLEX_FAMILIES]
    names += list(_HANDLE_FUNCS) + list(_EXTRA)
    return names


def lib():
    """Load librocsolver_b200.so and declare all entry points.  Raises if the library
    has not been built (python -m rocsolver_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m rocsolver_b200.build`")
    l = _c.CDLL(LIB_PATH)
    for p in "sdcz":
        for fam, args in _SIG.items():
            if p in "cz" and fam not in _COMPLEX_FAMILIES:
                continue
            f = getattr(l, f"rocsolver_{p}{fam}")
            f.restype = _c.c_int
            f.argtypes = [H] + args
    for name, (res, args) in list(_HANDLE_FUNCS.items()) + list(_EXTRA.items()):
        f = getattr(l, name)
        f.restype = res
        f.argtypes = args
    _lib = l
    return l


class Handle:
    """rocblas_handle bound to a CUDA stream (torch's current stream by default)."""

    def __init__(self, stream=None):
        self.h = H()
        st = lib().rocblas_create_handle(_c.byref(self.h))
        if st != SUCCESS:
            raise RuntimeError(f"rocblas_create_handle: {STATUS_NAMES[st]}")
        if stream is not None:
            self.set_stream(stream)

    def set_stream(self, stream):
        ptr = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", 0)
        lib().rocblas_set_stream(self.h, _c.c_void_p(ptr))

    def close(self):
        if self.h:
            lib().rocblas_destroy_handle(self.h)
            self.h = H()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def value(self):
        return self.h


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return None
    return _c.c_void_p(t.data_ptr())


def call(name, *args):
    """Call an exported entry point by name; returns the rocblas_status as int."""
    return getattr(lib(), name)(*args)


def check(status, what=""):
    if status != SUCCESS:
        raise RuntimeError(f"{what}: rocblas_status_{STATUS_NAMES[status]}")


def tuning_table():
    """The active kernel configuration table as text (tuning.h format)."""
    l = lib()
    size = l.rocsolver_b200_tuning_get(None, 0)
    buf = _c.create_string_buffer(size)
    l.rocsolver_b200_tuning_get(buf, size)
    return buf.value.decode()


def set_tuning_table(text):
    """Replace the active kernel configuration table; returns the rocblas status."""
    return lib().rocsolver_b200_tuning_set(text.encode())
