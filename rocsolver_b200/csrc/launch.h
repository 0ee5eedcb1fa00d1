// launch.h -- host-side launchers of the factor/solve kernels (internal interface between
// the C-ABI layer in api.cu and the CUDA translation units).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rocsolver.h"
#include "common.cuh"

namespace rsb {

// Every launcher returns success, not_implemented (size outside the supported range)
// or internal_error (launch failure).  None synchronises or allocates.
// tc (FP32 with pivoting only): trailing updates as split-TF32 tensor products
template <typename T>
rocblas_status launch_getrf(cudaStream_t s, int m, int n, Batch<T> A, int lda, int* ipiv,
                            int64_t strideP, int* info, int bc, bool pivot,
                            Gate gate = no_gate(), bool tc = false);
template <typename T>
rocblas_status launch_getrs(cudaStream_t s, int trans, int n, int nrhs, Batch<T> A, int lda,
                            const int* ipiv, int64_t strideP, Batch<T> B, int ldb,
                            const int* skip_info, int bc, Gate gate = no_gate());
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
// getrs (trans N) tuned for many right-hand sides (getri)
template <typename T>
rocblas_status launch_getrs_many(cudaStream_t s, int n, int nrhs, Batch<T> A, int lda,
                                 const int* ipiv, int64_t strideP, Batch<T> B, int ldb,
                                 const int* skip_info, int bc);

// the complex precisions (complex.cu); getrs takes trans 2 = conjugate transpose
#define RSB_DECLARE_COMPLEX_LAUNCHERS(C)                                                      \
    template <>                                                                               \
    rocblas_status launch_getrf<C>(cudaStream_t, int, int, Batch<C>, int, int*, int64_t, int*,\
                                   int, bool, Gate, bool);                                    \
    template <>                                                                               \
    rocblas_status launch_getrs<C>(cudaStream_t, int, int, int, Batch<C>, int, const int*,    \
                                   int64_t, Batch<C>, int, const int*, int, Gate);            \
    template <>                                                                               \
    rocblas_status launch_gesv<C>(cudaStream_t, int, int, Batch<C>, int, int*, int64_t,       \
                                  Batch<C>, int, int*, int);                                  \
    template <>                                                                               \
    rocblas_status launch_potrf<C>(cudaStream_t, int, int, Batch<C>, int, int*, int);         \
    template <>                                                                               \
    rocblas_status launch_potrs<C>(cudaStream_t, int, int, int, Batch<C>, int, Batch<C>, int, \
                                   const int*, int);
RSB_DECLARE_COMPLEX_LAUNCHERS(rocblas_float_complex)
RSB_DECLARE_COMPLEX_LAUNCHERS(rocblas_double_complex)
#undef RSB_DECLARE_COMPLEX_LAUNCHERS

// inverse from the LU factors (getri.cu): C.base == C.ptrs == nullptr means in place (the
// inverse is formed in ws, getri_workspace bytes, and copied over A where info == 0);
// ipiv == nullptr means no pivoting (npvt forms)
template <typename T>
size_t getri_workspace(int n, int bc, bool inplace);
template <typename T>
rocblas_status launch_getri(cudaStream_t s, int n, Batch<T> A, int lda, const int* ipiv,
                            int64_t strideP, Batch<T> C, int ldc, int* info, int bc, void* ws);

// mixed-precision solver (mixed.cu)
size_t dsgesv_workspace(int n, int nrhs, int bc);
rocblas_status launch_dsgesv(cudaStream_t s, int n, int nrhs, Batch<double> A, int lda,
                             int* ipiv, int64_t strideP, Batch<double> B, int ldb,
                             Batch<double> X, int ldx, int* iter, int* info, int bc, void* ws);
// adjoint of the batched solve (adjoint.cu); kind 0 = LU, 1 = Cholesky lower, 2 = upper
template <typename T>
rocblas_status launch_solve_adjoint(cudaStream_t s, int kind, int n, int nrhs, Batch<T> A,
                                    int lda, const int* ipiv, int64_t strideP, Batch<T> X,
                                    int ldx, Batch<T> G, int ldg, Batch<T> GA, int ldga,
                                    Batch<T> GB, int ldgb, int bc);

// variable-size batches (vbatched.cu); mode 0 gesv, 1 getrf, 2 getrs
size_t vbatched_workspace(int bc);
template <typename T>
rocblas_status launch_vbatched(cudaStream_t s, int mode, const int* n, const int* nrhs,
                               T* const* A, const int* lda, int* const* ipiv, T* const* B,
                               const int* ldb, int* info, int max_n, int max_nrhs, int bc,
                               void* ws);

// sets two int arrays to zero (quick returns)
rocblas_status launch_reset_info2(cudaStream_t s, int* a, int* b, int bc);

// largest m (rows) the CTA-resident LU / Cholesky kernels support
constexpr int MAX_CTA_ROWS = 2048;

} // namespace rsb
