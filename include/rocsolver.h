/* rocsolver-b200: B200 (sm_100a) implementation of rocSOLVER's batched dense
 * LU / Cholesky factor-and-solve path, exported under the reference's C ABI.
 *
 * The types below restate the subset of rocBLAS's public types that the
 * rocSOLVER prototypes use (library/src/include/rocblas.hpp:17-36 names the
 * status codes; rocsolver-extra-types.h:13-20 the layer flags).  The numeric
 * values are rocBLAS's public-header values so that a program compiled against
 * the real headers passes the same integers.
 *
 * Conventions (identical to the reference, library/include/rocsolver/rocsolver-functions.h):
 *   - matrices are column-major, element (i,j) at A[i + j*lda];
 *   - strided batches: member b starts at A + b*strideA (strides in elements, int64);
 *   - pointer-array batches: member b is A[b] (device array of device pointers);
 *   - ipiv is 1-based, ipiv[b*strideP + k] = row swapped with row k+1;
 *   - info[b] = 0 on success, k > 0 when U(k,k) is exactly zero (getrf) or the
 *     leading minor of order k is not positive (potrf);
 *   - every call is asynchronous on the handle's stream and never synchronises,
 *     so sequences of calls can be captured into a CUDA graph.
 * All array arguments are device memory owned by the caller.
 */
#ifndef ROCSOLVER_B200_ROCSOLVER_H
#define ROCSOLVER_B200_ROCSOLVER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define ROCSOLVER_EXPORT
#else
#define ROCSOLVER_EXPORT __attribute__((visibility("default")))
#endif

/* ---- rocBLAS shim types ------------------------------------------------ */
typedef int32_t rocblas_int;
typedef int64_t rocblas_stride;
typedef struct _rocblas_handle* rocblas_handle;
typedef uint32_t rocblas_layer_mode_flags;
/* complex element types, layout-compatible with the reference's (interleaved re, im) */
typedef struct
{
    float x, y;
} rocblas_float_complex;
typedef struct
{
    double x, y;
} rocblas_double_complex;

typedef enum rocblas_status_
{
    rocblas_status_success = 0,
    rocblas_status_invalid_handle = 1,
    rocblas_status_not_implemented = 2,
    rocblas_status_invalid_pointer = 3,
    rocblas_status_invalid_size = 4,
    rocblas_status_memory_error = 5,
    rocblas_status_internal_error = 6,
    rocblas_status_perf_degraded = 7,
    rocblas_status_size_query_mismatch = 8,
    rocblas_status_size_increased = 9,
    rocblas_status_size_unchanged = 10,
    rocblas_status_invalid_value = 11,
    rocblas_status_continue = 12,
    rocblas_status_check_numerics_fail = 13
} rocblas_status;

typedef enum rocblas_operation_
{
    rocblas_operation_none = 111,
    rocblas_operation_transpose = 112,
    rocblas_operation_conjugate_transpose = 113
} rocblas_operation;

typedef enum rocblas_fill_
{
    rocblas_fill_upper = 121,
    rocblas_fill_lower = 122,
    rocblas_fill_full = 123
} rocblas_fill;

/* ---- handle shim ---------------------------------------------------------
 * A handle is {CUDA stream, device workspace, size-query state}.  Creating a
 * handle makes no CUDA call; the workspace is allocated on first need (or is
 * supplied by the user with rocblas_set_workspace).  Semantics follow the
 * rocBLAS memory model exercised by clients/gtest/memory_model_gtest.cpp:54-170:
 * 32 MiB nominal reservation, ROCBLAS_DEVICE_MEMORY_SIZE makes the size
 * user-fixed, and a size query returns size_increased/size_unchanged instead
 * of computing. */
ROCSOLVER_EXPORT rocblas_status rocblas_create_handle(rocblas_handle* handle);
ROCSOLVER_EXPORT rocblas_status rocblas_destroy_handle(rocblas_handle handle);
/* stream is a cudaStream_t passed as void* (0 = legacy default stream) */
ROCSOLVER_EXPORT rocblas_status rocblas_set_stream(rocblas_handle handle, void* stream);
ROCSOLVER_EXPORT rocblas_status rocblas_get_stream(rocblas_handle handle, void** stream);
ROCSOLVER_EXPORT rocblas_status rocblas_start_device_memory_size_query(rocblas_handle handle);
ROCSOLVER_EXPORT rocblas_status rocblas_stop_device_memory_size_query(rocblas_handle handle,
                                                                      size_t* size);
ROCSOLVER_EXPORT int rocblas_is_device_memory_size_query(rocblas_handle handle);
ROCSOLVER_EXPORT int rocblas_is_managing_device_memory(rocblas_handle handle);
ROCSOLVER_EXPORT rocblas_status rocblas_get_device_memory_size(rocblas_handle handle,
                                                               size_t* size);
/* size 0 returns to library-managed memory; otherwise allocates exactly size bytes */
ROCSOLVER_EXPORT rocblas_status rocblas_set_device_memory_size(rocblas_handle handle,
                                                               size_t size);
/* user-owned device workspace (addr may be NULL with size 0 to return to managed mode) */
ROCSOLVER_EXPORT rocblas_status rocblas_set_workspace(rocblas_handle handle, void* addr,
                                                      size_t size);

/* library version, mirrors library/src/common/buildinfo.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_get_version_string(char* buf, size_t len);
ROCSOLVER_EXPORT rocblas_status rocsolver_get_version_string_size(size_t* len);

/* ---- multi-level logging ------------------------------------------------
 * Replaces rocsolver-functions.h:66-119 (library/src/common/rocsolver_logger.cpp).
 * rocsolver_log_begin opens a session whose layer mode and depth come from ROCSOLVER_LAYER
 * (bit mask: rocblas_layer_mode_log_trace 1, _log_bench 2, _log_profile 4; 0x10 adds
 * kernel launches) and ROCSOLVER_LEVELS (default 1); logs go to stderr, or to the files
 * named by ROCSOLVER_LOG_PATH / ROCSOLVER_LOG_{TRACE,BENCH,PROFILE}_PATH.  Every entry point
 * then writes a rocsolver-bench command line (bench), its trace tree (trace) or its
 * accumulated time (profile; this waits for the handle's stream on return, so do not enable
 * it while capturing a stream).  All return internal_error without an open session, and
 * rocsolver_log_begin with one already open. */
#define rocblas_layer_mode_none 0u
#define rocblas_layer_mode_log_trace 1u
#define rocblas_layer_mode_log_bench 2u
#define rocblas_layer_mode_log_profile 4u
#define rocblas_layer_mode_ex_log_kernel 0x10u
ROCSOLVER_EXPORT rocblas_status rocsolver_log_begin(void);
ROCSOLVER_EXPORT rocblas_status rocsolver_log_end(void);
ROCSOLVER_EXPORT rocblas_status rocsolver_log_set_layer_mode(const rocblas_layer_mode_flags layer_mode);
ROCSOLVER_EXPORT rocblas_status rocsolver_log_set_max_levels(const rocblas_int max_levels);
ROCSOLVER_EXPORT rocblas_status rocsolver_log_restore_defaults(void);
ROCSOLVER_EXPORT rocblas_status rocsolver_log_write_profile(void);
ROCSOLVER_EXPORT rocblas_status rocsolver_log_flush_profile(void);

/* ---- hot path: LU / Cholesky factor and solve ---------------------------
 * Each prototype keeps the reference's argument order and meaning exactly;
 * the comment names the reference declaration it replaces
 * (library/include/rocsolver/rocsolver-functions.h) and its implementation
 * file (library/src/lapack/).  Argument checks follow the reference order:
 * invalid_handle, invalid_value (enums), invalid_size, [size query],
 * invalid_pointer, then quick return. */
/* replaces rocsolver-functions.h:5139-5155 / lapack/roclapack_getrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrf(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_int* info);

/* replaces rocsolver-functions.h:5227-5247 / lapack/roclapack_getrf_batched.cpp:96-124 */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrf_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    float* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:5329-5349 / lapack/roclapack_getrf_strided_batched.cpp:94-122 */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrf_strided_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:4609-4622 / lapack/roclapack_getrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrf_npvt(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:4688-4702 / lapack/roclapack_getrf_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrf_npvt_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    float* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:4775-4790 / lapack/roclapack_getrf_strided_batched.cpp:154-208 */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrf_npvt_strided_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8562-8580 / lapack/roclapack_getrs.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrs(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    const rocblas_int* ipiv,
    float* B,
    const rocblas_int ldb);

/* replaces rocsolver-functions.h:8657-8680 / lapack/roclapack_getrs_batched.cpp:75 */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrs_batched(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* const A[],
    const rocblas_int lda,
    const rocblas_int* ipiv,
    const rocblas_stride strideP,
    float* const B[],
    const rocblas_int ldb,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8771-8796 / lapack/roclapack_getrs_strided_batched.cpp:74-108 */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrs_strided_batched(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    const rocblas_int* ipiv,
    const rocblas_stride strideP,
    float* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8872-8890 / lapack/roclapack_gesv.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgesv(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    float* B,
    const rocblas_int ldb,
    rocblas_int* info);

/* replaces rocsolver-functions.h:8970-8992 / lapack/roclapack_gesv_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgesv_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    float* const B[],
    const rocblas_int ldb,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9095-9108 / lapack/roclapack_gesv_strided_batched.cpp:92-127 */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgesv_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    float* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10188-10201 / lapack/roclapack_potrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_spotrf(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:10261-10276 / lapack/roclapack_potrf_batched.cpp:86 */
ROCSOLVER_EXPORT rocblas_status rocsolver_spotrf_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    float* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10340-10356 / lapack/roclapack_potrf_strided_batched.cpp:84-110 */
ROCSOLVER_EXPORT rocblas_status rocsolver_spotrf_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10426-10443 / lapack/roclapack_potrs.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_spotrs(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    float* B,
    const rocblas_int ldb);

/* replaces rocsolver-functions.h:10520-10538 / lapack/roclapack_potrs_batched.cpp:72 */
ROCSOLVER_EXPORT rocblas_status rocsolver_spotrs_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* const A[],
    const rocblas_int lda,
    float* const B[],
    const rocblas_int ldb,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10619-10642 / lapack/roclapack_potrs_strided_batched.cpp:71-102 */
ROCSOLVER_EXPORT rocblas_status rocsolver_spotrs_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    float* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10718-10736 / lapack/roclapack_posv.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sposv(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    float* B,
    const rocblas_int ldb,
    rocblas_int* info);

/* replaces rocsolver-functions.h:10816-10833 / lapack/roclapack_posv_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sposv_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* const A[],
    const rocblas_int lda,
    float* const B[],
    const rocblas_int ldb,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10931-10944 / lapack/roclapack_posv_strided_batched.cpp:87 */
ROCSOLVER_EXPORT rocblas_status rocsolver_sposv_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    float* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:5139-5155 / lapack/roclapack_getrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrf(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_int* info);

/* replaces rocsolver-functions.h:5227-5247 / lapack/roclapack_getrf_batched.cpp:96-124 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrf_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    double* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:5329-5349 / lapack/roclapack_getrf_strided_batched.cpp:94-122 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrf_strided_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:4609-4622 / lapack/roclapack_getrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrf_npvt(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:4688-4702 / lapack/roclapack_getrf_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrf_npvt_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    double* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:4775-4790 / lapack/roclapack_getrf_strided_batched.cpp:154-208 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrf_npvt_strided_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8562-8580 / lapack/roclapack_getrs.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrs(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    const rocblas_int* ipiv,
    double* B,
    const rocblas_int ldb);

/* replaces rocsolver-functions.h:8657-8680 / lapack/roclapack_getrs_batched.cpp:75 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrs_batched(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* const A[],
    const rocblas_int lda,
    const rocblas_int* ipiv,
    const rocblas_stride strideP,
    double* const B[],
    const rocblas_int ldb,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8771-8796 / lapack/roclapack_getrs_strided_batched.cpp:74-108 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrs_strided_batched(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    const rocblas_int* ipiv,
    const rocblas_stride strideP,
    double* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8872-8890 / lapack/roclapack_gesv.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgesv(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    double* B,
    const rocblas_int ldb,
    rocblas_int* info);

/* replaces rocsolver-functions.h:8970-8992 / lapack/roclapack_gesv_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgesv_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    double* const B[],
    const rocblas_int ldb,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9095-9108 / lapack/roclapack_gesv_strided_batched.cpp:92-127 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgesv_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    double* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10188-10201 / lapack/roclapack_potrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dpotrf(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:10261-10276 / lapack/roclapack_potrf_batched.cpp:86 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dpotrf_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    double* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10340-10356 / lapack/roclapack_potrf_strided_batched.cpp:84-110 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dpotrf_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10426-10443 / lapack/roclapack_potrs.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dpotrs(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    double* B,
    const rocblas_int ldb);

/* replaces rocsolver-functions.h:10520-10538 / lapack/roclapack_potrs_batched.cpp:72 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dpotrs_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* const A[],
    const rocblas_int lda,
    double* const B[],
    const rocblas_int ldb,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10619-10642 / lapack/roclapack_potrs_strided_batched.cpp:71-102 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dpotrs_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    double* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10718-10736 / lapack/roclapack_posv.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dposv(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    double* B,
    const rocblas_int ldb,
    rocblas_int* info);

/* replaces rocsolver-functions.h:10816-10833 / lapack/roclapack_posv_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dposv_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* const A[],
    const rocblas_int lda,
    double* const B[],
    const rocblas_int ldb,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10931-10944 / lapack/roclapack_posv_strided_batched.cpp:87 */
ROCSOLVER_EXPORT rocblas_status rocsolver_dposv_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    double* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    rocblas_int* info,
    const rocblas_int batch_count);

/* ---- complex precisions (c = rocblas_float_complex, z = rocblas_double_complex) --------
 * The same argument lists as the s / d forms; transposed solves accept
 * rocblas_operation_conjugate_transpose (op(A) = A^H), Cholesky factors a Hermitian
 * positive definite matrix (A = L L^H or U^H U). */
/* replaces rocsolver-functions.h:5155 / lapack/roclapack_getrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetrf(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_int* info);

/* replaces rocsolver-functions.h:5248 / lapack/roclapack_getrf_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetrf_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:5351 / lapack/roclapack_getrf_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetrf_strided_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:4623 / lapack/roclapack_getrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetrf_npvt(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:4703 / lapack/roclapack_getrf_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetrf_npvt_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:4791 / lapack/roclapack_getrf_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetrf_npvt_strided_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8582 / lapack/roclapack_getrs.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetrs(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_int* ipiv,
    rocblas_float_complex* B,
    const rocblas_int ldb);

/* replaces rocsolver-functions.h:8681 / lapack/roclapack_getrs_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetrs_batched(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    const rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_float_complex* const B[],
    const rocblas_int ldb,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8796 / lapack/roclapack_getrs_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetrs_strided_batched(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    const rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_float_complex* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8892 / lapack/roclapack_gesv.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgesv(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_float_complex* B,
    const rocblas_int ldb,
    rocblas_int* info);

/* replaces rocsolver-functions.h:8992 / lapack/roclapack_gesv_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgesv_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_float_complex* const B[],
    const rocblas_int ldb,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9109 / lapack/roclapack_gesv_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgesv_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_float_complex* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10202 / lapack/roclapack_potrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cpotrf(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:10276 / lapack/roclapack_potrf_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cpotrf_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10358 / lapack/roclapack_potrf_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cpotrf_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10444 / lapack/roclapack_potrs.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cpotrs(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_float_complex* B,
    const rocblas_int ldb);

/* replaces rocsolver-functions.h:10537 / lapack/roclapack_potrs_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cpotrs_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    rocblas_float_complex* const B[],
    const rocblas_int ldb,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10644 / lapack/roclapack_potrs_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cpotrs_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_float_complex* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10738 / lapack/roclapack_posv.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cposv(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_float_complex* B,
    const rocblas_int ldb,
    rocblas_int* info);

/* replaces rocsolver-functions.h:10834 / lapack/roclapack_posv_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cposv_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    rocblas_float_complex* const B[],
    const rocblas_int ldb,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10944 / lapack/roclapack_posv_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cposv_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_float_complex* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:5163 / lapack/roclapack_getrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetrf(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_int* info);

/* replaces rocsolver-functions.h:5258 / lapack/roclapack_getrf_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetrf_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:5362 / lapack/roclapack_getrf_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetrf_strided_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:4630 / lapack/roclapack_getrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetrf_npvt(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:4711 / lapack/roclapack_getrf_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetrf_npvt_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:4800 / lapack/roclapack_getrf_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetrf_npvt_strided_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8592 / lapack/roclapack_getrs.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetrs(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_int* ipiv,
    rocblas_double_complex* B,
    const rocblas_int ldb);

/* replaces rocsolver-functions.h:8693 / lapack/roclapack_getrs_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetrs_batched(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    const rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_double_complex* const B[],
    const rocblas_int ldb,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8810 / lapack/roclapack_getrs_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetrs_strided_batched(rocblas_handle handle,
    const rocblas_operation trans,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    const rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_double_complex* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:8902 / lapack/roclapack_gesv.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgesv(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_double_complex* B,
    const rocblas_int ldb,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9004 / lapack/roclapack_gesv_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgesv_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_double_complex* const B[],
    const rocblas_int ldb,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9123 / lapack/roclapack_gesv_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgesv_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_double_complex* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10209 / lapack/roclapack_potrf.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zpotrf(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:10284 / lapack/roclapack_potrf_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zpotrf_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10367 / lapack/roclapack_potrf_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zpotrf_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10453 / lapack/roclapack_potrs.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zpotrs(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_double_complex* B,
    const rocblas_int ldb);

/* replaces rocsolver-functions.h:10547 / lapack/roclapack_potrs_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zpotrs_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    rocblas_double_complex* const B[],
    const rocblas_int ldb,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10656 / lapack/roclapack_potrs_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zpotrs_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_double_complex* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10748 / lapack/roclapack_posv.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zposv(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_double_complex* B,
    const rocblas_int ldb,
    rocblas_int* info);

/* replaces rocsolver-functions.h:10845 / lapack/roclapack_posv_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zposv_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    rocblas_double_complex* const B[],
    const rocblas_int ldb,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:10957 / lapack/roclapack_posv_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zposv_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_double_complex* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    rocblas_int* info,
    const rocblas_int batch_count);

/* ---- inverse from the LU factors and the out-of-place solve --------------------
 * getri: A (the LU factors and ipiv from getrf) is overwritten by inv(A) where info = 0;
 * info = i > 0 when U(i,i) is the first zero diagonal entry, and A keeps its factors.
 * getri_outofplace: C = inv(A), A unchanged.  npvt forms: factors from getrf_npvt.
 * In-place getri needs n*n elements of workspace per member (handle workspace).
 * gesv_outofplace: X = A^{-1} B with A overwritten by its LU factors; B unchanged. */
/* replaces rocsolver-functions.h:9173-9186 / lapack/roclapack_getri.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri(rocblas_handle handle,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9245-9262 / lapack/roclapack_getri_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_batched(rocblas_handle handle,
    const rocblas_int n,
    float* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9329-9348 / lapack/roclapack_getri_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9402-9413 / lapack/roclapack_getri.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_npvt(rocblas_handle handle,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9463-9476 / lapack/roclapack_getri_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_npvt_batched(rocblas_handle handle,
    const rocblas_int n,
    float* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9532-9547 / lapack/roclapack_getri_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_npvt_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21380-21396 / lapack/roclapack_getri_outofplace.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_outofplace(rocblas_handle handle,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    float* C,
    const rocblas_int ldc,
    rocblas_int* info);

/* replaces rocsolver-functions.h:21462-21483 / lapack/roclapack_getri_outofplace_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_outofplace_batched(rocblas_handle handle,
    const rocblas_int n,
    float* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    float* const C[],
    const rocblas_int ldc,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21562-21588 / lapack/roclapack_getri_outofplace_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_outofplace_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    float* C,
    const rocblas_int ldc,
    const rocblas_stride strideC,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21653-21667 / lapack/roclapack_getri_outofplace.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_npvt_outofplace(rocblas_handle handle,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    float* C,
    const rocblas_int ldc,
    rocblas_int* info);

/* replaces rocsolver-functions.h:21725-21741 / lapack/roclapack_getri_outofplace_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_npvt_outofplace_batched(rocblas_handle handle,
    const rocblas_int n,
    float* const A[],
    const rocblas_int lda,
    float* const C[],
    const rocblas_int ldc,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21813-21834 / lapack/roclapack_getri_outofplace_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetri_npvt_outofplace_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    float* C,
    const rocblas_int ldc,
    const rocblas_stride strideC,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces lapack/roclapack_gesv_outofplace.cpp:106-119 (exported, not in the public header) */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgesv_outofplace(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    float* B,
    const rocblas_int ldb,
    float* X,
    const rocblas_int ldx,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9173-9186 / lapack/roclapack_getri.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri(rocblas_handle handle,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9245-9262 / lapack/roclapack_getri_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_batched(rocblas_handle handle,
    const rocblas_int n,
    double* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9329-9348 / lapack/roclapack_getri_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9402-9413 / lapack/roclapack_getri.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_npvt(rocblas_handle handle,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9463-9476 / lapack/roclapack_getri_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_npvt_batched(rocblas_handle handle,
    const rocblas_int n,
    double* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9532-9547 / lapack/roclapack_getri_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_npvt_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21380-21396 / lapack/roclapack_getri_outofplace.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_outofplace(rocblas_handle handle,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    double* C,
    const rocblas_int ldc,
    rocblas_int* info);

/* replaces rocsolver-functions.h:21462-21483 / lapack/roclapack_getri_outofplace_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_outofplace_batched(rocblas_handle handle,
    const rocblas_int n,
    double* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    double* const C[],
    const rocblas_int ldc,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21562-21588 / lapack/roclapack_getri_outofplace_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_outofplace_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    double* C,
    const rocblas_int ldc,
    const rocblas_stride strideC,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21653-21667 / lapack/roclapack_getri_outofplace.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_npvt_outofplace(rocblas_handle handle,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    double* C,
    const rocblas_int ldc,
    rocblas_int* info);

/* replaces rocsolver-functions.h:21725-21741 / lapack/roclapack_getri_outofplace_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_npvt_outofplace_batched(rocblas_handle handle,
    const rocblas_int n,
    double* const A[],
    const rocblas_int lda,
    double* const C[],
    const rocblas_int ldc,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21813-21834 / lapack/roclapack_getri_outofplace_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetri_npvt_outofplace_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    double* C,
    const rocblas_int ldc,
    const rocblas_stride strideC,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces lapack/roclapack_gesv_outofplace.cpp:121-135 (exported, not in the public header) */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgesv_outofplace(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    double* B,
    const rocblas_int ldb,
    double* X,
    const rocblas_int ldx,
    rocblas_int* info);

/* complex getri and gesv_outofplace: the same argument lists as the s / d forms above */
/* replaces rocsolver-functions.h:9187 / lapack/roclapack_getri.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9263 / lapack/roclapack_getri_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9349 / lapack/roclapack_getri_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9414 / lapack/roclapack_getri.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_npvt(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9477 / lapack/roclapack_getri_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_npvt_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9548 / lapack/roclapack_getri_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_npvt_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21398 / lapack/roclapack_getri_outofplace.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_outofplace(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_float_complex* C,
    const rocblas_int ldc,
    rocblas_int* info);

/* replaces rocsolver-functions.h:21484 / lapack/roclapack_getri_outofplace_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_outofplace_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_float_complex* const C[],
    const rocblas_int ldc,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21590 / lapack/roclapack_getri_outofplace_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_outofplace_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_float_complex* C,
    const rocblas_int ldc,
    const rocblas_stride strideC,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21669 / lapack/roclapack_getri_outofplace.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_npvt_outofplace(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_float_complex* C,
    const rocblas_int ldc,
    rocblas_int* info);

/* replaces rocsolver-functions.h:21744 / lapack/roclapack_getri_outofplace_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_npvt_outofplace_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* const A[],
    const rocblas_int lda,
    rocblas_float_complex* const C[],
    const rocblas_int ldc,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21837 / lapack/roclapack_getri_outofplace_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgetri_npvt_outofplace_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_float_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_float_complex* C,
    const rocblas_int ldc,
    const rocblas_stride strideC,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces lapack/roclapack_gesv_outofplace.cpp:137-151 (exported, not in the public header) */
ROCSOLVER_EXPORT rocblas_status rocsolver_cgesv_outofplace(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_float_complex* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_float_complex* B,
    const rocblas_int ldb,
    rocblas_float_complex* X,
    const rocblas_int ldx,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9194 / lapack/roclapack_getri.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9272 / lapack/roclapack_getri_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9359 / lapack/roclapack_getri_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9420 / lapack/roclapack_getri.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_npvt(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_int* info);

/* replaces rocsolver-functions.h:9484 / lapack/roclapack_getri_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_npvt_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:9556 / lapack/roclapack_getri_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_npvt_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21407 / lapack/roclapack_getri_outofplace.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_outofplace(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_double_complex* C,
    const rocblas_int ldc,
    rocblas_int* info);

/* replaces rocsolver-functions.h:21495 / lapack/roclapack_getri_outofplace_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_outofplace_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_double_complex* const C[],
    const rocblas_int ldc,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21604 / lapack/roclapack_getri_outofplace_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_outofplace_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_double_complex* C,
    const rocblas_int ldc,
    const rocblas_stride strideC,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21677 / lapack/roclapack_getri_outofplace.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_npvt_outofplace(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_double_complex* C,
    const rocblas_int ldc,
    rocblas_int* info);

/* replaces rocsolver-functions.h:21754 / lapack/roclapack_getri_outofplace_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_npvt_outofplace_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* const A[],
    const rocblas_int lda,
    rocblas_double_complex* const C[],
    const rocblas_int ldc,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces rocsolver-functions.h:21849 / lapack/roclapack_getri_outofplace_strided_batched.cpp */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgetri_npvt_outofplace_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    rocblas_double_complex* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_double_complex* C,
    const rocblas_int ldc,
    const rocblas_stride strideC,
    rocblas_int* info,
    const rocblas_int batch_count);

/* replaces lapack/roclapack_gesv_outofplace.cpp:153-167 (exported, not in the public header) */
ROCSOLVER_EXPORT rocblas_status rocsolver_zgesv_outofplace(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    rocblas_double_complex* A,
    const rocblas_int lda,
    rocblas_int* ipiv,
    rocblas_double_complex* B,
    const rocblas_int ldb,
    rocblas_double_complex* X,
    const rocblas_int ldx,
    rocblas_int* info);

/* ---- entry points with no counterpart in the reference ------------------ */

/* FP32 LU with partial pivoting for a strided batch whose trailing updates run on the
 * tensor cores as split-TF32 products (each operand split into two TF32 parts, three
 * products accumulated in FP32: FP32-level accuracy, rounding not identical to
 * rocsolver_sgetrf_strided_batched, so near-tied pivots may differ).  Arguments, ipiv and
 * info as rocsolver_sgetrf_strided_batched (library/src/lapack/roclapack_getrf.cpp).  This
 * is the factorisation rocsolver_dsgesv_strided_batched runs on its FP32 copy of A. */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrf_tf32_strided_batched(rocblas_handle handle,
    const rocblas_int m,
    const rocblas_int n,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    rocblas_int* info,
    const rocblas_int batch_count);

/* Mixed-precision solver with iterative refinement for a strided batch (LAPACK dsgesv
 * semantics per member; the reference has no mixed-precision gesv).  Each member is
 * factored in FP32 (LU with partial pivoting of an FP32 copy of A), then refined in FP64:
 * r = B - A X is formed from the FP64 A, the correction is solved with the FP32 factors,
 * and the loop stops when every column satisfies ||r||_inf <= ||x||_inf ||A||_inf eps
 * sqrt(n) (eps = 2^-53), after at most 10 corrections.
 *   X (ldx >= n)  : solution; B is not modified.
 *   iter[b] >= 0  : number of corrections; A unchanged; ipiv holds the FP32 pivots.
 *   iter[b] < 0   : refinement failed or was skipped (-1 not attempted, -2 FP32 overflow,
 *                   -3 FP32 factor singular, -11 no convergence in 10 corrections); the
 *                   member was re-solved in FP64: A holds its LU factors, ipiv/info come
 *                   from the FP64 factorisation.
 *   info[b]       : 0, or k > 0 if U(k,k) of the FP64 factorisation is exactly zero (then
 *                   X is not computed).
 * Uses the handle's device workspace: 4*n*n*batch_count bytes plus O(batch_count). */
ROCSOLVER_EXPORT rocblas_status rocsolver_dsgesv_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    rocblas_int* ipiv,
    const rocblas_stride strideP,
    double* B,
    const rocblas_int ldb,
    const rocblas_stride strideB,
    double* X,
    const rocblas_int ldx,
    const rocblas_stride strideX,
    rocblas_int* iter,
    rocblas_int* info,
    const rocblas_int batch_count);

/* Adjoint of the batched solve X = A^{-1} B (no counterpart in the reference).  From the
 * getrf factors of A (A, lda, strideA, ipiv, strideP as returned by getrf) and the upstream
 * gradient G = dL/dX, computes gB = A^{-T} G and gA = -gB X^T without refactoring.
 * gB may alias G.  X is the forward solution (ldx >= n). */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrs_adjoint_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    const rocblas_int* ipiv,
    const rocblas_stride strideP,
    float* X,
    const rocblas_int ldx,
    const rocblas_stride strideX,
    float* G,
    const rocblas_int ldg,
    const rocblas_stride strideG,
    float* gA,
    const rocblas_int ldga,
    const rocblas_stride strideGA,
    float* gB,
    const rocblas_int ldgb,
    const rocblas_stride strideGB,
    const rocblas_int batch_count);

/* Same for the SPD solve with potrf factors (uplo as given to potrf): gB = A^{-1} G,
 * gA = -gB X^T (unsymmetrised gradient with respect to every entry of A). */
ROCSOLVER_EXPORT rocblas_status rocsolver_spotrs_adjoint_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    float* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    float* X,
    const rocblas_int ldx,
    const rocblas_stride strideX,
    float* G,
    const rocblas_int ldg,
    const rocblas_stride strideG,
    float* gA,
    const rocblas_int ldga,
    const rocblas_stride strideGA,
    float* gB,
    const rocblas_int ldgb,
    const rocblas_stride strideGB,
    const rocblas_int batch_count);

/* Variable-size batches in one persistent launch (no counterpart in the reference).
 * n, nrhs, lda, ldb are DEVICE arrays of batch_count entries; A, B, ipiv are device
 * arrays of device pointers; max_n / max_nrhs (host) bound every member and select the
 * kernel configuration.  Members are ordered by size on the device (largest first) and
 * pulled from a work queue; no host synchronisation, so a call can be captured into a
 * CUDA graph once the handle's workspace is large enough (call once, or size-query and
 * rocblas_set_workspace, before capturing).  A member whose sizes are out of range gets
 * info = -1 and is not touched.  gesv/getrf: same per-member semantics as the
 * fixed-size routines (square members). */
ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrf_vbatched(rocblas_handle handle,
    const rocblas_int* n,
    float* const A[],
    const rocblas_int* lda,
    rocblas_int* const ipiv[],
    rocblas_int* info,
    const rocblas_int max_n,
    const rocblas_int batch_count);

ROCSOLVER_EXPORT rocblas_status rocsolver_sgetrs_vbatched(rocblas_handle handle,
    const rocblas_int* n,
    const rocblas_int* nrhs,
    float* const A[],
    const rocblas_int* lda,
    rocblas_int* const ipiv[],
    float* const B[],
    const rocblas_int* ldb,
    const rocblas_int max_n,
    const rocblas_int max_nrhs,
    const rocblas_int batch_count);

ROCSOLVER_EXPORT rocblas_status rocsolver_sgesv_vbatched(rocblas_handle handle,
    const rocblas_int* n,
    const rocblas_int* nrhs,
    float* const A[],
    const rocblas_int* lda,
    rocblas_int* const ipiv[],
    float* const B[],
    const rocblas_int* ldb,
    rocblas_int* info,
    const rocblas_int max_n,
    const rocblas_int max_nrhs,
    const rocblas_int batch_count);

/* Adjoint of the batched solve X = A^{-1} B (no counterpart in the reference).  From the
 * getrf factors of A (A, lda, strideA, ipiv, strideP as returned by getrf) and the upstream
 * gradient G = dL/dX, computes gB = A^{-T} G and gA = -gB X^T without refactoring.
 * gB may alias G.  X is the forward solution (ldx >= n). */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrs_adjoint_strided_batched(rocblas_handle handle,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    const rocblas_int* ipiv,
    const rocblas_stride strideP,
    double* X,
    const rocblas_int ldx,
    const rocblas_stride strideX,
    double* G,
    const rocblas_int ldg,
    const rocblas_stride strideG,
    double* gA,
    const rocblas_int ldga,
    const rocblas_stride strideGA,
    double* gB,
    const rocblas_int ldgb,
    const rocblas_stride strideGB,
    const rocblas_int batch_count);

/* Same for the SPD solve with potrf factors (uplo as given to potrf): gB = A^{-1} G,
 * gA = -gB X^T (unsymmetrised gradient with respect to every entry of A). */
ROCSOLVER_EXPORT rocblas_status rocsolver_dpotrs_adjoint_strided_batched(rocblas_handle handle,
    const rocblas_fill uplo,
    const rocblas_int n,
    const rocblas_int nrhs,
    double* A,
    const rocblas_int lda,
    const rocblas_stride strideA,
    double* X,
    const rocblas_int ldx,
    const rocblas_stride strideX,
    double* G,
    const rocblas_int ldg,
    const rocblas_stride strideG,
    double* gA,
    const rocblas_int ldga,
    const rocblas_stride strideGA,
    double* gB,
    const rocblas_int ldgb,
    const rocblas_stride strideGB,
    const rocblas_int batch_count);

/* Variable-size batches in one persistent launch (no counterpart in the reference).
 * n, nrhs, lda, ldb are DEVICE arrays of batch_count entries; A, B, ipiv are device
 * arrays of device pointers; max_n / max_nrhs (host) bound every member and select the
 * kernel configuration.  Members are ordered by size on the device (largest first) and
 * pulled from a work queue; no host synchronisation, so a call can be captured into a
 * CUDA graph once the handle's workspace is large enough (call once, or size-query and
 * rocblas_set_workspace, before capturing).  A member whose sizes are out of range gets
 * info = -1 and is not touched.  gesv/getrf: same per-member semantics as the
 * fixed-size routines (square members). */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrf_vbatched(rocblas_handle handle,
    const rocblas_int* n,
    double* const A[],
    const rocblas_int* lda,
    rocblas_int* const ipiv[],
    rocblas_int* info,
    const rocblas_int max_n,
    const rocblas_int batch_count);

ROCSOLVER_EXPORT rocblas_status rocsolver_dgetrs_vbatched(rocblas_handle handle,
    const rocblas_int* n,
    const rocblas_int* nrhs,
    double* const A[],
    const rocblas_int* lda,
    rocblas_int* const ipiv[],
    double* const B[],
    const rocblas_int* ldb,
    const rocblas_int max_n,
    const rocblas_int max_nrhs,
    const rocblas_int batch_count);

ROCSOLVER_EXPORT rocblas_status rocsolver_dgesv_vbatched(rocblas_handle handle,
    const rocblas_int* n,
    const rocblas_int* nrhs,
    double* const A[],
    const rocblas_int* lda,
    rocblas_int* const ipiv[],
    double* const B[],
    const rocblas_int* ldb,
    rocblas_int* info,
    const rocblas_int max_n,
    const rocblas_int max_nrhs,
    const rocblas_int batch_count);

/* Variable-size gesv that never allocates device memory (no counterpart in the
 * reference).  Same arguments and per-member results as rocsolver_dgesv_vbatched.  That
 * routine takes a little scratch (its work list) from the handle's workspace, which the
 * library allocates with cudaMalloc on first use; callers that may not allocate (code
 * running while a memory pool owns the device memory, allocation-free real-time loops,
 * plugins whose host framework forbids device allocations) use this variant, which keeps
 * the scratch in a fixed ~4 MiB array in the library's device memory (held on each GPU
 * where it has been called, until the process exits).
 *   - batch_count is limited to 1048576 members; larger batches return invalid_size.
 *   - All calls share the array: calls that overlap on the GPU race; order them on one
 *     stream.  Nothing carries over between calls (the work list is rebuilt each call).
 *   - The first call on a device looks up the array's device address.  Under CUDA's lazy
 *     module loading (the default since CUDA 12.2) that is when the driver places the
 *     array on the device, so make the first call (a warm-up with batch_count > 0) before
 *     a memory pool claims the device's free memory, and before any stream capture on
 *     that device. */
ROCSOLVER_EXPORT rocblas_status rocsolver_dgesv_vbatched_noalloc(rocblas_handle handle,
    const rocblas_int* n,
    const rocblas_int* nrhs,
    double* const A[],
    const rocblas_int* lda,
    rocblas_int* const ipiv[],
    double* const B[],
    const rocblas_int* ldb,
    rocblas_int* info,
    const rocblas_int max_n,
    const rocblas_int max_nrhs,
    const rocblas_int batch_count);

/* ---- Kernel configuration table (no counterpart in the reference, whose block sizes and
 * kernel switch points are compile-time constants: library/src/include/ideal_sizes.hpp:
 * 166-240, docs/design/tuning.rst:20-31).  The table is text, one entry per line:
 *   getrf    <s|d|t> <m_max> <threads> <rows_per_thread> <panel_width> <chunk> <fold>
 *   vbatched <s|d> <n_max> <threads> <rows_per_thread> <panel_width> <chunk> <fold> <ctas_per_sm>
 * (t: the FP32 LU with split-TF32 updates of sgetrf_tf32 and dsgesv; without t entries it
 * uses the s entries; fold = 2 in a t entry runs its trailing updates on the tcgen05 tensor
 * cores).  It is written by the autotuner (python -m rocsolver_b200.tune) and read when the first
 * handle is created, from $ROCSOLVER_B200_TUNING or else tuning_b200.txt beside the
 * library.  Entries that name an unavailable configuration fall back to the built-in
 * choice; results do not depend on the table, only speed does. */
ROCSOLVER_EXPORT rocblas_status rocsolver_b200_tuning_set(const char* text);   /* replace */
ROCSOLVER_EXPORT rocblas_status rocsolver_b200_tuning_load(const char* path);  /* from file */
/* Writes the active table (NUL-terminated, truncated to len) and returns its full size
 * including the NUL. */
ROCSOLVER_EXPORT size_t rocsolver_b200_tuning_get(char* buf, size_t len);

/* ---- Bounds-checked build (no counterpart in the reference's API; its debug aid is the
 * ROCSOLVER_VERIFY_ASSUMPTIONS build, library/src/include/lib_host_helpers.hpp:63-80).
 * librocsolver_b200_checked.so (python -m rocsolver_b200.build --checked) checks every
 * element access of the factor and solve kernels against the matrix dimensions and every
 * pivot index against 1..n; a violation is counted and recorded instead of performed.
 * result[0..3] receives the number of violations since the last call and the first one's
 * source line and indices, and the record is cleared.  The call synchronises with the
 * device.  The normal library returns rocblas_status_not_implemented. */
ROCSOLVER_EXPORT rocblas_status rocsolver_b200_bounds_check(rocblas_int* result);

#ifdef __cplusplus
}
#endif

#endif /* ROCSOLVER_B200_ROCSOLVER_H */
