// api.cu -- extern "C" entry points with the reference's names, argument order and
// argument-check order.  Each *_impl restates the reference's _impl + argCheck pair:
//   getrf : lapack/roclapack_getrf_strided_batched.cpp:8-84, roclapack_getf2.hpp:489-517
//   getrs : lapack/roclapack_getrs_strided_batched.cpp:8-72, roclapack_getrs.hpp:17-49
//   gesv  : lapack/roclapack_gesv_strided_batched.cpp:8-90, roclapack_gesv.hpp:18-47,105-178
//   potrf : lapack/roclapack_potrf_strided_batched.cpp:8-82, roclapack_potf2.hpp:107-134
//   potrs : lapack/roclapack_potrs_strided_batched.cpp:8-70, roclapack_potrs.hpp:17-46
//   posv  : lapack/roclapack_posv_strided_batched.cpp, roclapack_posv.hpp:18-47,101-170
//   getri : lapack/roclapack_getri_strided_batched.cpp, roclapack_getri.hpp:233-260
//   getri_outofplace : lapack/roclapack_getri_outofplace*.cpp,
//                      roclapack_getri_outofplace.hpp:39-68
//   gesv_outofplace  : lapack/roclapack_gesv_outofplace.cpp:15-100,
//                      roclapack_gesv_outofplace.hpp:10-40,112-170
// Order of checks: invalid_handle, invalid_value (enum arguments), invalid_size, then a
// device-memory size query returns here, then invalid_pointer, then quick returns.
#include "handle.h"
#include "launch.h"
#include "logger.h"

using namespace rsb;

namespace {

inline bool bad_op(rocblas_operation t)
{
    return t != rocblas_operation_none && t != rocblas_operation_transpose
           && t != rocblas_operation_conjugate_transpose;
}
inline bool bad_fill(rocblas_fill f)
{
    return f != rocblas_fill_upper && f != rocblas_fill_lower;
}

template <typename T>
struct is_complex
{
    static constexpr bool value = false;
};
template <>
struct is_complex<rocblas_float_complex>
{
    static constexpr bool value = true;
};
template <>
struct is_complex<rocblas_double_complex>
{
    static constexpr bool value = true;
};

template <typename T>
rocblas_status getrf_impl(rocblas_handle h, int m, int n, Batch<T> A, const void* Aptr, int lda,
                          int* ipiv, int64_t strideP, int* info, int bc, bool pivot,
                          bool tc = false)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(m < 0 || n < 0 || lda < m || bc < 0)
        return rocblas_status_invalid_size;
    if(h->querying)
        return ws_query(h, 0);
    const int64_t mn = (int64_t)m * n;
    if((mn && !Aptr) || (mn && pivot && !ipiv) || (bc && !info))
        return rocblas_status_invalid_pointer;
    if(bc == 0)
        return rocblas_status_success;
    if(m == 0 || n == 0)
        return launch_reset_info(h->stream, info, bc);
    RSB_LOG_STEP(pivot ? "getrf" : "getrf_npvt", logging::arg("m", m), logging::arg("n", n),
                 logging::arg("lda", lda), logging::arg("bc", bc));
    return launch_getrf<T>(h->stream, m, n, A, lda, ipiv, strideP, info, bc, pivot, no_gate(),
                           tc);
}

template <typename T>
rocblas_status getrs_impl(rocblas_handle h, rocblas_operation trans, int n, int nrhs,
                          Batch<T> A, const void* Aptr, int lda, const int* ipiv,
                          int64_t strideP, Batch<T> B, const void* Bptr, int ldb, int bc)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(bad_op(trans))
        return rocblas_status_invalid_value;
    if(n < 0 || nrhs < 0 || lda < n || ldb < n || bc < 0)
        return rocblas_status_invalid_size;
    if(h->querying)
        return ws_query(h, 0);
    if((n && !Aptr) || (n && !ipiv) || (nrhs && n && !Bptr))
        return rocblas_status_invalid_pointer;
    if(n == 0 || nrhs == 0 || bc == 0)
        return rocblas_status_success;
    RSB_LOG_STEP("getrs", logging::arg("trans", trans), logging::arg("n", n), logging::arg("nrhs", nrhs),
                 logging::arg("lda", lda), logging::arg("ldb", ldb), logging::arg("bc", bc));
    // 0 = N, 1 = T, 2 = C; for the real types C is T
    const int t = trans == rocblas_operation_none        ? 0
                  : trans == rocblas_operation_transpose || !is_complex<T>::value ? 1
                                                                                  : 2;
    return launch_getrs<T>(h->stream, t, n, nrhs, A, lda, ipiv, strideP, B, ldb, nullptr, bc);
}

template <typename T>
rocblas_status gesv_impl(rocblas_handle h, int n, int nrhs, Batch<T> A, const void* Aptr,
                         int lda, int* ipiv, int64_t strideP, Batch<T> B, const void* Bptr,
                         int ldb, int* info, int bc)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(n < 0 || nrhs < 0 || lda < n || ldb < n || bc < 0)
        return rocblas_status_invalid_size;
    if(h->querying)
        return ws_query(h, 0);
    if((n && !Aptr) || (n && !ipiv) || (nrhs && n && !Bptr) || (bc && !info))
        return rocblas_status_invalid_pointer;
    if(bc == 0)
        return rocblas_status_success;
    // the reference zeroes info and returns without factoring when A or B is empty
    if(n == 0 || nrhs == 0)
        return launch_reset_info(h->stream, info, bc);
    RSB_LOG_STEP("gesv", logging::arg("n", n), logging::arg("nrhs", nrhs), logging::arg("lda", lda),
                 logging::arg("ldb", ldb), logging::arg("bc", bc));
    return launch_gesv<T>(h->stream, n, nrhs, A, lda, ipiv, strideP, B, ldb, info, bc);
}

template <typename T>
rocblas_status potrf_impl(rocblas_handle h, rocblas_fill uplo, int n, Batch<T> A,
                          const void* Aptr, int lda, int* info, int bc)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(bad_fill(uplo))
        return rocblas_status_invalid_value;
    if(n < 0 || lda < n || bc < 0)
        return rocblas_status_invalid_size;
    if(h->querying)
        return ws_query(h, 0);
    if((n && !Aptr) || (bc && !info))
        return rocblas_status_invalid_pointer;
    if(bc == 0)
        return rocblas_status_success;
    if(n == 0)
        return launch_reset_info(h->stream, info, bc);
    RSB_LOG_STEP("potrf", logging::arg("uplo", uplo), logging::arg("n", n), logging::arg("lda", lda),
                 logging::arg("bc", bc));
    return launch_potrf<T>(h->stream, uplo == rocblas_fill_upper, n, A, lda, info, bc);
}

template <typename T>
rocblas_status potrs_impl(rocblas_handle h, rocblas_fill uplo, int n, int nrhs, Batch<T> A,
                          const void* Aptr, int lda, Batch<T> B, const void* Bptr, int ldb,
                          int bc)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(bad_fill(uplo))
        return rocblas_status_invalid_value;
    if(n < 0 || nrhs < 0 || lda < n || ldb < n || bc < 0)
        return rocblas_status_invalid_size;
    if(h->querying)
        return ws_query(h, 0);
    if((n && !Aptr) || (nrhs && n && !Bptr))
        return rocblas_status_invalid_pointer;
    if(n == 0 || nrhs == 0 || bc == 0)
        return rocblas_status_success;
    RSB_LOG_STEP("potrs", logging::arg("uplo", uplo), logging::arg("n", n), logging::arg("nrhs", nrhs),
                 logging::arg("lda", lda), logging::arg("ldb", ldb), logging::arg("bc", bc));
    return launch_potrs<T>(h->stream, uplo == rocblas_fill_upper, n, nrhs, A, lda, B, ldb,
                           nullptr, bc);
}

template <typename T>
rocblas_status posv_impl(rocblas_handle h, rocblas_fill uplo, int n, int nrhs, Batch<T> A,
                         const void* Aptr, int lda, Batch<T> B, const void* Bptr, int ldb,
                         int* info, int bc)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(bad_fill(uplo))
        return rocblas_status_invalid_value;
    if(n < 0 || nrhs < 0 || lda < n || ldb < n || bc < 0)
        return rocblas_status_invalid_size;
    if(h->querying)
        return ws_query(h, 0);
    if((n && !Aptr) || (nrhs && n && !Bptr) || (bc && !info))
        return rocblas_status_invalid_pointer;
    if(bc == 0)
        return rocblas_status_success;
    if(n == 0 || nrhs == 0)
        return launch_reset_info(h->stream, info, bc);
    const int up = uplo == rocblas_fill_upper;
    RSB_LOG_STEP("posv", logging::arg("uplo", uplo), logging::arg("n", n), logging::arg("nrhs", nrhs),
                 logging::arg("lda", lda), logging::arg("ldb", ldb), logging::arg("bc", bc));
    rocblas_status st = launch_potrf<T>(h->stream, up, n, A, lda, info, bc);
    if(st != rocblas_status_success)
        return st;
    return launch_potrs<T>(h->stream, up, n, nrhs, A, lda, B, ldb, info, bc);
}

// getri (C == nullptr: in place) and getri_outofplace; pivot == false: the npvt forms
template <typename T>
rocblas_status getri_impl(rocblas_handle h, int n, Batch<T> A, const void* Aptr, int lda,
                          int* ipiv, int64_t strideP, Batch<T> C, const void* Cptr, int ldc,
                          int* info, int bc, bool pivot, bool outofplace)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(n < 0 || lda < n || (outofplace && ldc < n) || bc < 0)
        return rocblas_status_invalid_size;
    const size_t ws_bytes = (n && bc) ? getri_workspace<T>(n, bc, !outofplace) : 0;
    if(h->querying)
        return ws_query(h, ws_bytes);
    if((n && !Aptr) || (outofplace && n && !Cptr) || (n && pivot && !ipiv) || (bc && !info))
        return rocblas_status_invalid_pointer;
    if(bc == 0)
        return rocblas_status_success;
    if(n == 0)
        return launch_reset_info(h->stream, info, bc);
    void* ws = nullptr;
    rocblas_status st = ws_get(h, ws_bytes, &ws);
    if(st != rocblas_status_success)
        return st;
    RSB_LOG_STEP(outofplace ? "getri_outofplace" : "getri", logging::arg("n", n),
                 logging::arg("lda", lda), logging::arg("bc", bc));
    return launch_getri<T>(h->stream, n, A, lda, pivot ? ipiv : nullptr, strideP,
                           outofplace ? C : Batch<T>{nullptr, nullptr, 0}, ldc, info, bc, ws);
}

// gesv_outofplace: X = B, then gesv on (A, X); B is not modified, X keeps the copy of B for
// a singular A (the reference leaves X undefined there)
template <typename T>
rocblas_status gesv_outofplace_impl(rocblas_handle h, int n, int nrhs, T* A, int lda, int* ipiv,
                                    T* B, int ldb, T* X, int ldx, int* info)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(n < 0 || nrhs < 0 || lda < n || ldb < n || ldx < n)
        return rocblas_status_invalid_size;
    if(h->querying)
        return ws_query(h, 0);
    if((n && !A) || (n && !ipiv) || (nrhs && n && !B) || (nrhs && n && !X)
       || !info)
        return rocblas_status_invalid_pointer;
    if(n == 0 || nrhs == 0)
        return launch_reset_info(h->stream, info, 1);
    RSB_LOG_STEP("gesv_outofplace", logging::arg("n", n), logging::arg("nrhs", nrhs),
                 logging::arg("lda", lda), logging::arg("ldb", ldb), logging::arg("ldx", ldx));
    if(cudaMemcpy2DAsync(X, sizeof(T) * (size_t)ldx, B, sizeof(T) * (size_t)ldb,
                         sizeof(T) * (size_t)n, nrhs, cudaMemcpyDeviceToDevice, h->stream)
       != cudaSuccess)
        return rocblas_status_internal_error;
    return launch_gesv<T>(h->stream, n, nrhs, strided<T>(A, 0), lda, ipiv, 0, strided<T>(X, 0),
                          ldx, info, 1);
}

rocblas_status dsgesv_impl(rocblas_handle h, int n, int nrhs, double* A, int lda,
                           int64_t strideA, int* ipiv, int64_t strideP, double* B, int ldb,
                           int64_t strideB, double* X, int ldx, int64_t strideX, int* iter,
                           int* info, int bc)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(n < 0 || nrhs < 0 || lda < n || ldb < n || ldx < n || bc < 0)
        return rocblas_status_invalid_size;
    const size_t ws_bytes = (n && nrhs && bc) ? dsgesv_workspace(n, nrhs, bc) : 0;
    if(h->querying)
        return ws_query(h, ws_bytes);
    const int64_t nn = (int64_t)n * nrhs;
    if((n && !A) || (n && !ipiv) || (nn && !B) || (nn && !X) || (bc && !info) || (bc && !iter))
        return rocblas_status_invalid_pointer;
    if(bc == 0)
        return rocblas_status_success;
    if(n == 0 || nrhs == 0)
        return launch_reset_info2(h->stream, info, iter, bc);
    void* ws = nullptr;
    rocblas_status st = ws_get(h, ws_bytes, &ws);
    if(st != rocblas_status_success)
        return st;
    RSB_LOG_STEP("dsgesv", logging::arg("n", n), logging::arg("nrhs", nrhs), logging::arg("lda", lda),
                 logging::arg("ldb", ldb), logging::arg("ldx", ldx), logging::arg("bc", bc));
    return launch_dsgesv(h->stream, n, nrhs, strided<double>(A, strideA), lda, ipiv, strideP,
                         strided<double>(B, strideB), ldb, strided<double>(X, strideX), ldx, iter,
                         info, bc, ws);
}

template <typename T>
rocblas_status adjoint_impl(rocblas_handle h, int kind, int n, int nrhs, T* A, int lda,
                            int64_t sA, const int* ipiv, int64_t sP, T* X, int ldx, int64_t sX,
                            T* G, int ldg, int64_t sG, T* gA, int ldga, int64_t sGA, T* gB,
                            int ldgb, int64_t sGB, int bc)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(n < 0 || nrhs < 0 || lda < n || ldx < n || ldg < n || ldga < n || ldgb < n || bc < 0)
        return rocblas_status_invalid_size;
    if(h->querying)
        return ws_query(h, 0);
    const int64_t nn = (int64_t)n * nrhs;
    if((n && !A) || (kind == 0 && n && !ipiv) || (nn && (!X || !G || !gB)) || (n && !gA))
        return rocblas_status_invalid_pointer;
    if(n == 0 || bc == 0)
        return rocblas_status_success;
    RSB_LOG_STEP(kind == 0 ? "getrs_adjoint" : "potrs_adjoint", logging::arg("n", n),
                 logging::arg("nrhs", nrhs), logging::arg("lda", lda), logging::arg("bc", bc));
    return launch_solve_adjoint<T>(h->stream, kind, n, nrhs, strided<T>(A, sA), lda, ipiv, sP,
                                   strided<T>(X, sX), ldx, strided<T>(G, sG), ldg,
                                   strided<T>(gA, sGA), ldga, strided<T>(gB, sGB), ldgb, bc);
}

template <typename T>
rocblas_status vbatched_impl(rocblas_handle h, int mode, const int* n, const int* nrhs,
                             T* const* A, const int* lda, int* const* ipiv, T* const* B,
                             const int* ldb, int* info, int max_n, int max_nrhs, int bc)
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(max_n < 0 || max_nrhs < 0 || bc < 0)
        return rocblas_status_invalid_size;
    const size_t ws_bytes = bc ? vbatched_workspace(bc) : 0;
    if(h->querying)
        return ws_query(h, ws_bytes);
    if(bc && (!n || !A || !lda || !ipiv || (mode != 2 && !info)))
        return rocblas_status_invalid_pointer;
    if(bc && mode != 1 && (!nrhs || !B || !ldb))
        return rocblas_status_invalid_pointer;
    if(bc == 0)
        return rocblas_status_success;
    void* ws = nullptr;
    rocblas_status st = ws_get(h, ws_bytes, &ws);
    if(st != rocblas_status_success)
        return st;
    RSB_LOG_STEP(mode == 0 ? "gesv_vbatched" : mode == 1 ? "getrf_vbatched" : "getrs_vbatched",
                 logging::arg("max_n", max_n), logging::arg("max_nrhs", max_nrhs), logging::arg("bc", bc));
    return launch_vbatched<T>(h->stream, mode, n, nrhs, A, lda, ipiv, B, ldb, info,
                              max_n > 0 ? max_n : 1, max_nrhs, bc, ws);
}

} // namespace

#define RSB_API_NEW(P, T)                                                                       \
    rocblas_status rocsolver_##P##getrs_adjoint_strided_batched(                                \
        rocblas_handle handle, const rocblas_int n, const rocblas_int nrhs, T* A,              \
        const rocblas_int lda, const rocblas_stride strideA, const rocblas_int* ipiv,          \
        const rocblas_stride strideP, T* X, const rocblas_int ldx, const rocblas_stride strideX,\
        T* G, const rocblas_int ldg, const rocblas_stride strideG, T* gA,                      \
        const rocblas_int ldga, const rocblas_stride strideGA, T* gB, const rocblas_int ldgb,  \
        const rocblas_stride strideGB, const rocblas_int batch_count)                          \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrs_adjoint_strided_batched", logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--strideP", strideP), logging::arg("--ldx", ldx), logging::arg("--ldg", ldg), logging::arg("--ldga", ldga), logging::arg("--ldgb", ldgb), logging::arg("--batch_count", batch_count));\
        return adjoint_impl<T>(handle, 0, n, nrhs, A, lda, strideA, ipiv, strideP, X, ldx,      \
                               strideX, G, ldg, strideG, gA, ldga, strideGA, gB, ldgb,          \
                               strideGB, batch_count);                                          \
    }                                                                                           \
    rocblas_status rocsolver_##P##potrs_adjoint_strided_batched(                                \
        rocblas_handle handle, const rocblas_fill uplo, const rocblas_int n,                   \
        const rocblas_int nrhs, T* A, const rocblas_int lda, const rocblas_stride strideA,     \
        T* X, const rocblas_int ldx, const rocblas_stride strideX, T* G, const rocblas_int ldg, \
        const rocblas_stride strideG, T* gA, const rocblas_int ldga,                           \
        const rocblas_stride strideGA, T* gB, const rocblas_int ldgb,                          \
        const rocblas_stride strideGB, const rocblas_int batch_count)                          \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "potrs_adjoint_strided_batched", logging::arg("--uplo", uplo), logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--ldx", ldx), logging::arg("--ldg", ldg), logging::arg("--ldga", ldga), logging::arg("--ldgb", ldgb), logging::arg("--batch_count", batch_count));\
        if(handle && bad_fill(uplo))                                                           \
            return rocblas_status_invalid_value;                                                \
        return adjoint_impl<T>(handle, uplo == rocblas_fill_upper ? 2 : 1, n, nrhs, A, lda,     \
                               strideA, nullptr, 0, X, ldx, strideX, G, ldg, strideG, gA, ldga, \
                               strideGA, gB, ldgb, strideGB, batch_count);                      \
    }                                                                                           \
    rocblas_status rocsolver_##P##getrf_vbatched(                                               \
        rocblas_handle handle, const rocblas_int* n, T* const A[], const rocblas_int* lda,     \
        rocblas_int* const ipiv[], rocblas_int* info, const rocblas_int max_n,                 \
        const rocblas_int batch_count)                                                         \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrf_vbatched", logging::arg("--max_n", max_n), logging::arg("--batch_count", batch_count));\
        return vbatched_impl<T>(handle, 1, n, nullptr, A, lda, ipiv, nullptr, nullptr, info,   \
                                max_n, 0, batch_count);                                         \
    }                                                                                           \
    rocblas_status rocsolver_##P##getrs_vbatched(                                               \
        rocblas_handle handle, const rocblas_int* n, const rocblas_int* nrhs, T* const A[],    \
        const rocblas_int* lda, rocblas_int* const ipiv[], T* const B[],                       \
        const rocblas_int* ldb, const rocblas_int max_n, const rocblas_int max_nrhs,           \
        const rocblas_int batch_count)                                                         \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrs_vbatched", logging::arg("--max_n", max_n), logging::arg("--max_nrhs", max_nrhs), logging::arg("--batch_count", batch_count));\
        return vbatched_impl<T>(handle, 2, n, nrhs, A, lda, ipiv, B, ldb, nullptr, max_n,      \
                                max_nrhs, batch_count);                                         \
    }                                                                                           \
    rocblas_status rocsolver_##P##gesv_vbatched(                                                \
        rocblas_handle handle, const rocblas_int* n, const rocblas_int* nrhs, T* const A[],    \
        const rocblas_int* lda, rocblas_int* const ipiv[], T* const B[],                       \
        const rocblas_int* ldb, rocblas_int* info, const rocblas_int max_n,                    \
        const rocblas_int max_nrhs, const rocblas_int batch_count)                             \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "gesv_vbatched", logging::arg("--max_n", max_n), logging::arg("--max_nrhs", max_nrhs), logging::arg("--batch_count", batch_count));\
        return vbatched_impl<T>(handle, 0, n, nrhs, A, lda, ipiv, B, ldb, info, max_n,         \
                                max_nrhs, batch_count);                                         \
    }

extern "C" {
RSB_API_NEW(s, float)
RSB_API_NEW(d, double)
}

extern "C" rocblas_status rocsolver_dsgesv_strided_batched(
    rocblas_handle handle, const rocblas_int n, const rocblas_int nrhs, double* A,
    const rocblas_int lda, const rocblas_stride strideA, rocblas_int* ipiv,
    const rocblas_stride strideP, double* B, const rocblas_int ldb, const rocblas_stride strideB,
    double* X, const rocblas_int ldx, const rocblas_stride strideX, rocblas_int* iter,
    rocblas_int* info, const rocblas_int batch_count)
{
    RSB_LOG_TOP('d', "dsgesv_strided_batched", logging::arg("-n", n), logging::arg("--nrhs", nrhs),
                logging::arg("--lda", lda), logging::arg("--strideA", strideA),
                logging::arg("--strideP", strideP), logging::arg("--ldb", ldb),
                logging::arg("--strideB", strideB), logging::arg("--ldx", ldx),
                logging::arg("--strideX", strideX), logging::arg("--batch_count", batch_count));
    return dsgesv_impl(handle, n, nrhs, A, lda, strideA, ipiv, strideP, B, ldb, strideB, X, ldx,
                       strideX, iter, info, batch_count);
}

// FP32 LU with split-TF32 tensor-core trailing updates (the factorisation of dsgesv);
// argument checks as getrf (lapack/roclapack_getrf_strided_batched.cpp:8-84)
extern "C" rocblas_status rocsolver_sgetrf_tf32_strided_batched(
    rocblas_handle handle, const rocblas_int m, const rocblas_int n, float* A,
    const rocblas_int lda, const rocblas_stride strideA, rocblas_int* ipiv,
    const rocblas_stride strideP, rocblas_int* info, const rocblas_int batch_count)
{
    RSB_LOG_TOP('s', "getrf_tf32_strided_batched", logging::arg("-m", m), logging::arg("-n", n),
                logging::arg("--lda", lda), logging::arg("--strideA", strideA),
                logging::arg("--strideP", strideP), logging::arg("--batch_count", batch_count));
    return getrf_impl<float>(handle, m, n, strided<float>(A, strideA), A, lda, ipiv, strideP,
                             info, batch_count, true, true);
}

#define RSB_API_TYPE(P, T)                                                                      \
    rocblas_status rocsolver_##P##getrf(rocblas_handle handle, const rocblas_int m,             \
                                        const rocblas_int n, T* A, const rocblas_int lda,      \
                                        rocblas_int* ipiv, rocblas_int* info)                  \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrf", logging::arg("-m", m), logging::arg("-n", n), logging::arg("--lda", lda));\
        return getrf_impl<T>(handle, m, n, strided<T>(A, 0), A, lda, ipiv, 0, info, 1, true);   \
    }                                                                                           \
    rocblas_status rocsolver_##P##getrf_batched(rocblas_handle handle, const rocblas_int m,     \
                                                const rocblas_int n, T* const A[],              \
                                                const rocblas_int lda, rocblas_int* ipiv,       \
                                                const rocblas_stride strideP, rocblas_int* info,\
                                                const rocblas_int batch_count)                  \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrf_batched", logging::arg("-m", m), logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--strideP", strideP), logging::arg("--batch_count", batch_count));\
        return getrf_impl<T>(handle, m, n, pointers<T>(A), A, lda, ipiv, strideP, info,         \
                             batch_count, true);                                                \
    }                                                                                           \
    rocblas_status rocsolver_##P##getrf_strided_batched(                                        \
        rocblas_handle handle, const rocblas_int m, const rocblas_int n, T* A,                 \
        const rocblas_int lda, const rocblas_stride strideA, rocblas_int* ipiv,                \
        const rocblas_stride strideP, rocblas_int* info, const rocblas_int batch_count)        \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrf_strided_batched", logging::arg("-m", m), logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--strideP", strideP), logging::arg("--batch_count", batch_count));\
        return getrf_impl<T>(handle, m, n, strided<T>(A, strideA), A, lda, ipiv, strideP,      \
                             info, batch_count, true);                                          \
    }                                                                                           \
    rocblas_status rocsolver_##P##getrf_npvt(rocblas_handle handle, const rocblas_int m,        \
                                             const rocblas_int n, T* A, const rocblas_int lda, \
                                             rocblas_int* info)                                 \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrf_npvt", logging::arg("-m", m), logging::arg("-n", n), logging::arg("--lda", lda));\
        return getrf_impl<T>(handle, m, n, strided<T>(A, 0), A, lda, nullptr, 0, info, 1,      \
                             false);                                                            \
    }                                                                                           \
    rocblas_status rocsolver_##P##getrf_npvt_batched(                                           \
        rocblas_handle handle, const rocblas_int m, const rocblas_int n, T* const A[],         \
        const rocblas_int lda, rocblas_int* info, const rocblas_int batch_count)               \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrf_npvt_batched", logging::arg("-m", m), logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--batch_count", batch_count));\
        return getrf_impl<T>(handle, m, n, pointers<T>(A), A, lda, nullptr, 0, info,            \
                             batch_count, false);                                               \
    }                                                                                           \
    rocblas_status rocsolver_##P##getrf_npvt_strided_batched(                                   \
        rocblas_handle handle, const rocblas_int m, const rocblas_int n, T* A,                 \
        const rocblas_int lda, const rocblas_stride strideA, rocblas_int* info,                \
        const rocblas_int batch_count)                                                          \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrf_npvt_strided_batched", logging::arg("-m", m), logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--batch_count", batch_count));\
        return getrf_impl<T>(handle, m, n, strided<T>(A, strideA), A, lda, nullptr, 0, info,   \
                             batch_count, false);                                               \
    }                                                                                           \
    rocblas_status rocsolver_##P##getrs(rocblas_handle handle, const rocblas_operation trans,   \
                                        const rocblas_int n, const rocblas_int nrhs, T* A,     \
                                        const rocblas_int lda, const rocblas_int* ipiv, T* B,  \
                                        const rocblas_int ldb)                                  \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrs", logging::arg("--trans", trans), logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--ldb", ldb));\
        return getrs_impl<T>(handle, trans, n, nrhs, strided<T>(A, 0), A, lda, ipiv, 0,         \
                             strided<T>(B, 0), B, ldb, 1);                                      \
    }                                                                                           \
    rocblas_status rocsolver_##P##getrs_batched(                                                \
        rocblas_handle handle, const rocblas_operation trans, const rocblas_int n,             \
        const rocblas_int nrhs, T* const A[], const rocblas_int lda, const rocblas_int* ipiv,  \
        const rocblas_stride strideP, T* const B[], const rocblas_int ldb,                     \
        const rocblas_int batch_count)                                                          \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrs_batched", logging::arg("--trans", trans), logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--strideP", strideP), logging::arg("--ldb", ldb), logging::arg("--batch_count", batch_count));\
        return getrs_impl<T>(handle, trans, n, nrhs, pointers<T>(A), A, lda, ipiv, strideP,     \
                             pointers<T>(B), B, ldb, batch_count);                              \
    }                                                                                           \
    rocblas_status rocsolver_##P##getrs_strided_batched(                                        \
        rocblas_handle handle, const rocblas_operation trans, const rocblas_int n,             \
        const rocblas_int nrhs, T* A, const rocblas_int lda, const rocblas_stride strideA,     \
        const rocblas_int* ipiv, const rocblas_stride strideP, T* B, const rocblas_int ldb,    \
        const rocblas_stride strideB, const rocblas_int batch_count)                           \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getrs_strided_batched", logging::arg("--trans", trans), logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--strideP", strideP), logging::arg("--ldb", ldb), logging::arg("--strideB", strideB), logging::arg("--batch_count", batch_count));\
        return getrs_impl<T>(handle, trans, n, nrhs, strided<T>(A, strideA), A, lda, ipiv,      \
                             strideP, strided<T>(B, strideB), B, ldb, batch_count);             \
    }                                                                                           \
    rocblas_status rocsolver_##P##gesv(rocblas_handle handle, const rocblas_int n,              \
                                       const rocblas_int nrhs, T* A, const rocblas_int lda,    \
                                       rocblas_int* ipiv, T* B, const rocblas_int ldb,         \
                                       rocblas_int* info)                                      \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "gesv", logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--ldb", ldb));\
        return gesv_impl<T>(handle, n, nrhs, strided<T>(A, 0), A, lda, ipiv, 0,                 \
                            strided<T>(B, 0), B, ldb, info, 1);                                 \
    }                                                                                           \
    rocblas_status rocsolver_##P##gesv_batched(                                                 \
        rocblas_handle handle, const rocblas_int n, const rocblas_int nrhs, T* const A[],      \
        const rocblas_int lda, rocblas_int* ipiv, const rocblas_stride strideP, T* const B[],  \
        const rocblas_int ldb, rocblas_int* info, const rocblas_int batch_count)               \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "gesv_batched", logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--strideP", strideP), logging::arg("--ldb", ldb), logging::arg("--batch_count", batch_count));\
        return gesv_impl<T>(handle, n, nrhs, pointers<T>(A), A, lda, ipiv, strideP,             \
                            pointers<T>(B), B, ldb, info, batch_count);                         \
    }                                                                                           \
    rocblas_status rocsolver_##P##gesv_strided_batched(                                         \
        rocblas_handle handle, const rocblas_int n, const rocblas_int nrhs, T* A,              \
        const rocblas_int lda, const rocblas_stride strideA, rocblas_int* ipiv,                \
        const rocblas_stride strideP, T* B, const rocblas_int ldb,                             \
        const rocblas_stride strideB, rocblas_int* info, const rocblas_int batch_count)        \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "gesv_strided_batched", logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--strideP", strideP), logging::arg("--ldb", ldb), logging::arg("--strideB", strideB), logging::arg("--batch_count", batch_count));\
        return gesv_impl<T>(handle, n, nrhs, strided<T>(A, strideA), A, lda, ipiv, strideP,     \
                            strided<T>(B, strideB), B, ldb, info, batch_count);                 \
    }                                                                                           \
    rocblas_status rocsolver_##P##potrf(rocblas_handle handle, const rocblas_fill uplo,         \
                                        const rocblas_int n, T* A, const rocblas_int lda,      \
                                        rocblas_int* info)                                      \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "potrf", logging::arg("--uplo", uplo), logging::arg("-n", n), logging::arg("--lda", lda));\
        return potrf_impl<T>(handle, uplo, n, strided<T>(A, 0), A, lda, info, 1);               \
    }                                                                                           \
    rocblas_status rocsolver_##P##potrf_batched(rocblas_handle handle, const rocblas_fill uplo, \
                                                const rocblas_int n, T* const A[],              \
                                                const rocblas_int lda, rocblas_int* info,       \
                                                const rocblas_int batch_count)                  \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "potrf_batched", logging::arg("--uplo", uplo), logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--batch_count", batch_count));\
        return potrf_impl<T>(handle, uplo, n, pointers<T>(A), A, lda, info, batch_count);       \
    }                                                                                           \
    rocblas_status rocsolver_##P##potrf_strided_batched(                                        \
        rocblas_handle handle, const rocblas_fill uplo, const rocblas_int n, T* A,             \
        const rocblas_int lda, const rocblas_stride strideA, rocblas_int* info,                \
        const rocblas_int batch_count)                                                          \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "potrf_strided_batched", logging::arg("--uplo", uplo), logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--batch_count", batch_count));\
        return potrf_impl<T>(handle, uplo, n, strided<T>(A, strideA), A, lda, info,             \
                             batch_count);                                                      \
    }                                                                                           \
    rocblas_status rocsolver_##P##potrs(rocblas_handle handle, const rocblas_fill uplo,         \
                                        const rocblas_int n, const rocblas_int nrhs, T* A,     \
                                        const rocblas_int lda, T* B, const rocblas_int ldb)    \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "potrs", logging::arg("--uplo", uplo), logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--ldb", ldb));\
        return potrs_impl<T>(handle, uplo, n, nrhs, strided<T>(A, 0), A, lda,                   \
                             strided<T>(B, 0), B, ldb, 1);                                      \
    }                                                                                           \
    rocblas_status rocsolver_##P##potrs_batched(                                                \
        rocblas_handle handle, const rocblas_fill uplo, const rocblas_int n,                   \
        const rocblas_int nrhs, T* const A[], const rocblas_int lda, T* const B[],             \
        const rocblas_int ldb, const rocblas_int batch_count)                                  \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "potrs_batched", logging::arg("--uplo", uplo), logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--ldb", ldb), logging::arg("--batch_count", batch_count));\
        return potrs_impl<T>(handle, uplo, n, nrhs, pointers<T>(A), A, lda, pointers<T>(B), B,  \
                             ldb, batch_count);                                                 \
    }                                                                                           \
    rocblas_status rocsolver_##P##potrs_strided_batched(                                        \
        rocblas_handle handle, const rocblas_fill uplo, const rocblas_int n,                   \
        const rocblas_int nrhs, T* A, const rocblas_int lda, const rocblas_stride strideA,     \
        T* B, const rocblas_int ldb, const rocblas_stride strideB,                             \
        const rocblas_int batch_count)                                                          \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "potrs_strided_batched", logging::arg("--uplo", uplo), logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--ldb", ldb), logging::arg("--strideB", strideB), logging::arg("--batch_count", batch_count));\
        return potrs_impl<T>(handle, uplo, n, nrhs, strided<T>(A, strideA), A, lda,             \
                             strided<T>(B, strideB), B, ldb, batch_count);                      \
    }                                                                                           \
    rocblas_status rocsolver_##P##posv(rocblas_handle handle, const rocblas_fill uplo,          \
                                       const rocblas_int n, const rocblas_int nrhs, T* A,      \
                                       const rocblas_int lda, T* B, const rocblas_int ldb,     \
                                       rocblas_int* info)                                      \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "posv", logging::arg("--uplo", uplo), logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--ldb", ldb));\
        return posv_impl<T>(handle, uplo, n, nrhs, strided<T>(A, 0), A, lda, strided<T>(B, 0),  \
                            B, ldb, info, 1);                                                   \
    }                                                                                           \
    rocblas_status rocsolver_##P##posv_batched(                                                 \
        rocblas_handle handle, const rocblas_fill uplo, const rocblas_int n,                   \
        const rocblas_int nrhs, T* const A[], const rocblas_int lda, T* const B[],             \
        const rocblas_int ldb, rocblas_int* info, const rocblas_int batch_count)               \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "posv_batched", logging::arg("--uplo", uplo), logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--ldb", ldb), logging::arg("--batch_count", batch_count));\
        return posv_impl<T>(handle, uplo, n, nrhs, pointers<T>(A), A, lda, pointers<T>(B), B,   \
                            ldb, info, batch_count);                                            \
    }                                                                                           \
    rocblas_status rocsolver_##P##posv_strided_batched(                                         \
        rocblas_handle handle, const rocblas_fill uplo, const rocblas_int n,                   \
        const rocblas_int nrhs, T* A, const rocblas_int lda, const rocblas_stride strideA,     \
        T* B, const rocblas_int ldb, const rocblas_stride strideB, rocblas_int* info,          \
        const rocblas_int batch_count)                                                          \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "posv_strided_batched", logging::arg("--uplo", uplo), logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--ldb", ldb), logging::arg("--strideB", strideB), logging::arg("--batch_count", batch_count));\
        return posv_impl<T>(handle, uplo, n, nrhs, strided<T>(A, strideA), A, lda,              \
                            strided<T>(B, strideB), B, ldb, info, batch_count);                 \
    }

#define RSB_API_GETRI(P, T)                                                                     \
    rocblas_status rocsolver_##P##getri(rocblas_handle handle, const rocblas_int n, T* A,       \
                                        const rocblas_int lda, rocblas_int* ipiv,              \
                                        rocblas_int* info)                                      \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri", logging::arg("-n", n), logging::arg("--lda", lda));             \
        return getri_impl<T>(handle, n, strided<T>(A, 0), A, lda, ipiv, 0,                      \
                             Batch<T>{nullptr, nullptr, 0}, nullptr, 0, info, 1, true, false);  \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_batched(                                                \
        rocblas_handle handle, const rocblas_int n, T* const A[], const rocblas_int lda,       \
        rocblas_int* ipiv, const rocblas_stride strideP, rocblas_int* info,                    \
        const rocblas_int batch_count)                                                          \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_batched", logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--strideP", strideP), logging::arg("--batch_count", batch_count));\
        return getri_impl<T>(handle, n, pointers<T>(A), A, lda, ipiv, strideP,                  \
                             Batch<T>{nullptr, nullptr, 0}, nullptr, 0, info, batch_count,      \
                             true, false);                                                      \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_strided_batched(                                        \
        rocblas_handle handle, const rocblas_int n, T* A, const rocblas_int lda,               \
        const rocblas_stride strideA, rocblas_int* ipiv, const rocblas_stride strideP,         \
        rocblas_int* info, const rocblas_int batch_count)                                      \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_strided_batched", logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--strideP", strideP), logging::arg("--batch_count", batch_count));\
        return getri_impl<T>(handle, n, strided<T>(A, strideA), A, lda, ipiv, strideP,          \
                             Batch<T>{nullptr, nullptr, 0}, nullptr, 0, info, batch_count,      \
                             true, false);                                                      \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_npvt(rocblas_handle handle, const rocblas_int n, T* A,  \
                                             const rocblas_int lda, rocblas_int* info)          \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_npvt", logging::arg("-n", n), logging::arg("--lda", lda));        \
        return getri_impl<T>(handle, n, strided<T>(A, 0), A, lda, nullptr, 0,                  \
                             Batch<T>{nullptr, nullptr, 0}, nullptr, 0, info, 1, false, false); \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_npvt_batched(rocblas_handle handle, const rocblas_int n,\
                                                     T* const A[], const rocblas_int lda,       \
                                                     rocblas_int* info,                         \
                                                     const rocblas_int batch_count)             \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_npvt_batched", logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--batch_count", batch_count));\
        return getri_impl<T>(handle, n, pointers<T>(A), A, lda, nullptr, 0,                     \
                             Batch<T>{nullptr, nullptr, 0}, nullptr, 0, info, batch_count,      \
                             false, false);                                                     \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_npvt_strided_batched(                                   \
        rocblas_handle handle, const rocblas_int n, T* A, const rocblas_int lda,               \
        const rocblas_stride strideA, rocblas_int* info, const rocblas_int batch_count)        \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_npvt_strided_batched", logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--batch_count", batch_count));\
        return getri_impl<T>(handle, n, strided<T>(A, strideA), A, lda, nullptr, 0,             \
                             Batch<T>{nullptr, nullptr, 0}, nullptr, 0, info, batch_count,      \
                             false, false);                                                     \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_outofplace(rocblas_handle handle, const rocblas_int n,  \
                                                   T* A, const rocblas_int lda,                 \
                                                   rocblas_int* ipiv, T* C,                     \
                                                   const rocblas_int ldc, rocblas_int* info)    \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_outofplace", logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--ldc", ldc));\
        return getri_impl<T>(handle, n, strided<T>(A, 0), A, lda, ipiv, 0, strided<T>(C, 0), C, \
                             ldc, info, 1, true, true);                                         \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_outofplace_batched(                                     \
        rocblas_handle handle, const rocblas_int n, T* const A[], const rocblas_int lda,       \
        rocblas_int* ipiv, const rocblas_stride strideP, T* const C[], const rocblas_int ldc,  \
        rocblas_int* info, const rocblas_int batch_count)                                      \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_outofplace_batched", logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--strideP", strideP), logging::arg("--ldc", ldc), logging::arg("--batch_count", batch_count));\
        return getri_impl<T>(handle, n, pointers<T>(A), A, lda, ipiv, strideP, pointers<T>(C),  \
                             C, ldc, info, batch_count, true, true);                            \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_outofplace_strided_batched(                             \
        rocblas_handle handle, const rocblas_int n, T* A, const rocblas_int lda,               \
        const rocblas_stride strideA, rocblas_int* ipiv, const rocblas_stride strideP, T* C,   \
        const rocblas_int ldc, const rocblas_stride strideC, rocblas_int* info,                \
        const rocblas_int batch_count)                                                          \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_outofplace_strided_batched", logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--strideP", strideP), logging::arg("--ldc", ldc), logging::arg("--strideC", strideC), logging::arg("--batch_count", batch_count));\
        return getri_impl<T>(handle, n, strided<T>(A, strideA), A, lda, ipiv, strideP,          \
                             strided<T>(C, strideC), C, ldc, info, batch_count, true, true);    \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_npvt_outofplace(rocblas_handle handle,                  \
                                                        const rocblas_int n, T* A,              \
                                                        const rocblas_int lda, T* C,            \
                                                        const rocblas_int ldc,                  \
                                                        rocblas_int* info)                      \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_npvt_outofplace", logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--ldc", ldc));\
        return getri_impl<T>(handle, n, strided<T>(A, 0), A, lda, nullptr, 0, strided<T>(C, 0), \
                             C, ldc, info, 1, false, true);                                     \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_npvt_outofplace_batched(                                \
        rocblas_handle handle, const rocblas_int n, T* const A[], const rocblas_int lda,       \
        T* const C[], const rocblas_int ldc, rocblas_int* info, const rocblas_int batch_count) \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_npvt_outofplace_batched", logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--ldc", ldc), logging::arg("--batch_count", batch_count));\
        return getri_impl<T>(handle, n, pointers<T>(A), A, lda, nullptr, 0, pointers<T>(C), C,  \
                             ldc, info, batch_count, false, true);                              \
    }                                                                                           \
    rocblas_status rocsolver_##P##getri_npvt_outofplace_strided_batched(                        \
        rocblas_handle handle, const rocblas_int n, T* A, const rocblas_int lda,               \
        const rocblas_stride strideA, T* C, const rocblas_int ldc, const rocblas_stride strideC,\
        rocblas_int* info, const rocblas_int batch_count)                                      \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "getri_npvt_outofplace_strided_batched", logging::arg("-n", n), logging::arg("--lda", lda), logging::arg("--strideA", strideA), logging::arg("--ldc", ldc), logging::arg("--strideC", strideC), logging::arg("--batch_count", batch_count));\
        return getri_impl<T>(handle, n, strided<T>(A, strideA), A, lda, nullptr, 0,             \
                             strided<T>(C, strideC), C, ldc, info, batch_count, false, true);   \
    }                                                                                           \
    rocblas_status rocsolver_##P##gesv_outofplace(                                              \
        rocblas_handle handle, const rocblas_int n, const rocblas_int nrhs, T* A,              \
        const rocblas_int lda, rocblas_int* ipiv, T* B, const rocblas_int ldb, T* X,           \
        const rocblas_int ldx, rocblas_int* info)                                               \
    {                                                                                           \
        RSB_LOG_TOP(#P[0], "gesv_outofplace", logging::arg("-n", n), logging::arg("--nrhs", nrhs), logging::arg("--lda", lda), logging::arg("--ldb", ldb), logging::arg("--ldx", ldx));\
        return gesv_outofplace_impl<T>(handle, n, nrhs, A, lda, ipiv, B, ldb, X, ldx, info);    \
    }

extern "C" {
RSB_API_TYPE(s, float)
RSB_API_TYPE(d, double)
RSB_API_TYPE(c, rocblas_float_complex)
RSB_API_TYPE(z, rocblas_double_complex)
RSB_API_GETRI(s, float)
RSB_API_GETRI(d, double)
RSB_API_GETRI(c, rocblas_float_complex)
RSB_API_GETRI(z, rocblas_double_complex)
}
