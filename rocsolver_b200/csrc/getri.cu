// getri.cu -- inverse of a general matrix from its LU factors (getri, getri_outofplace and
// their npvt forms).
//
// Replaces library/src/lapack/roclapack_getri.hpp:265-390 (rocsolver_getri_template: trtri of
// U, then inv(A) L = inv(U) by blocked GEMM/TRSM, then column interchanges) and
// roclapack_getri_outofplace.hpp:73-127 (check_singularity, C = I, getrs on C).
//
// B200 design: both forms solve A C = I with the library's getrs kernels (one warp per
// matrix and right-hand-side group for n <= 32, otherwise one CTA per matrix and group of
// four columns, the factors staged through inverted diagonal blocks), after one prep kernel
// that finds the first zero diagonal entry of U (info, LAPACK dtrtri's singularity test) and
// writes the identity into C.  In-place getri solves into the handle workspace and copies
// the inverse back over the factors of the members with info = 0; members with info > 0 keep
// their factors (LAPACK dgetri returns before touching A), and for getri_outofplace their C
// holds the identity (the reference leaves it undefined).
#include "handle.h"
#include "launch.h"
#include "logger.h"

namespace rsb {

// info[b] = first i (1-based) with U(i,i) == 0, else 0; W_b = I (n x n, ld ldw).  One CTA
// per member.
template <typename T>
__global__ void __launch_bounds__(256)
    getri_prep_kernel(int n, Batch<T> A, int lda, Batch<T> W, int ldw, int* info)
{
    __shared__ int first;
    const int64_t b = blockIdx.x;
    const T* a = A.at(b);
    T* w = W.at(b);
    if(threadIdx.x == 0)
        first = INT_MAX;
    __syncthreads();
    int mine = INT_MAX;
    for(int i = threadIdx.x; i < n; i += blockDim.x)
        if(a[ix(i, i, lda)] == T(0))
        {
            mine = i;
            break;
        }
    if(mine != INT_MAX)
        atomicMin(&first, mine);
    const int64_t total = (int64_t)n * n;
    for(int64_t e = threadIdx.x; e < total; e += blockDim.x)
    {
        const int i = (int)(e % n), j = (int)(e / n);
        w[ix(i, j, ldw)] = i == j ? T(1) : T(0);
    }
    __syncthreads();
    if(threadIdx.x == 0)
        info[b] = first == INT_MAX ? 0 : first + 1;
}

// A_b = W_b for the members with info[b] == 0
template <typename T>
__global__ void __launch_bounds__(256)
    getri_copy_back_kernel(int n, Batch<T> W, int ldw, Batch<T> A, int lda, const int* info)
{
    const int64_t b = blockIdx.x;
    if(info[b] != 0)
        return;
    const T* w = W.at(b);
    T* a = A.at(b);
    const int64_t total = (int64_t)n * n;
    for(int64_t e = threadIdx.x; e < total; e += blockDim.x)
    {
        const int i = (int)(e % n), j = (int)(e / n);
        a[ix(i, j, lda)] = w[ix(i, j, ldw)];
    }
}

size_t getri_workspace(int n, int bc, size_t elem, bool inplace)
{
    return inplace ? ws_round(elem * (size_t)n * n * bc) : 0;
}

template <typename T>
rocblas_status launch_getri(cudaStream_t s, int n, Batch<T> A, int lda, const int* ipiv,
                            int64_t strideP, Batch<T> C, int ldc, int* info, int bc, void* ws)
{
    const bool inplace = C.base == nullptr && C.ptrs == nullptr;
    Batch<T> W = inplace ? strided<T>(static_cast<T*>(ws), (int64_t)n * n) : C;
    const int ldw = inplace ? n : ldc;
    {
        RSB_LOG_KERNEL("getri_prep_kernel");
        getri_prep_kernel<T><<<bc, 256, 0, s>>>(n, A, lda, W, ldw, info);
    }
    if(cudaGetLastError() != cudaSuccess)
        return rocblas_status_internal_error;
    rocblas_status st = launch_getrs_many<T>(s, n, n, A, lda, ipiv, strideP, W, ldw, info, bc);
    if(st != rocblas_status_success || !inplace)
        return st;
    RSB_LOG_KERNEL("getri_copy_back_kernel");
    getri_copy_back_kernel<T><<<bc, 256, 0, s>>>(n, W, ldw, A, lda, info);
    return cudaGetLastError() == cudaSuccess ? rocblas_status_success
                                             : rocblas_status_internal_error;
}

template rocblas_status launch_getri<float>(cudaStream_t, int, Batch<float>, int, const int*,
                                            int64_t, Batch<float>, int, int*, int, void*);
template rocblas_status launch_getri<double>(cudaStream_t, int, Batch<double>, int, const int*,
                                             int64_t, Batch<double>, int, int*, int, void*);

} // namespace rsb
