// launch.h -- host-side launchers of the factor/solve kernels (internal interface between
// the C-ABI layer in api.cpp and the CUDA translation units).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rocsolver.h"
#include "common.cuh"

namespace rsb {

// Every launcher returns success, not_implemented (size outside the supported range)
// or internal_error (launch failure).  None synchronises or allocates.
template <typename T>
rocblas_status launch_getrf(cudaStream_t s, int m, int n, Batch<T> A, int lda, int* ipiv,
                            int64_t strideP, int* info, int bc, bool pivot);
template <typename T>
rocblas_status launch_getrs(cudaStream_t s, int trans, int n, int nrhs, Batch<T> A, int lda,
                            const int* ipiv, int64_t strideP, Batch<T> B, int ldb,
                            const int* skip_info, int bc);
template <typename T>
rocblas_status launch_gesv(cudaStream_t s, int n, int nrhs, Batch<T> A, int lda, int* ipiv,
                           int64_t strideP, Batch<T> B, int ldb, int* info, int bc);
template <typename T>
rocblas_status launch_potrf(cudaStream_t s, int upper, int n, Batch<T> A, int lda, int* info,
                            int bc);
template <typename T>
rocblas_status launch_potrs(cudaStream_t s, int upper, int n, int nrhs, Batch<T> A, int lda,
                            Batch<T> B, int ldb, const int* skip_info, int bc);
rocblas_status launch_reset_info(cudaStream_t s, int* info, int bc);

// largest m (rows) the CTA-resident LU / Cholesky kernels support
constexpr int MAX_CTA_ROWS = 2048;

} // namespace rsb
