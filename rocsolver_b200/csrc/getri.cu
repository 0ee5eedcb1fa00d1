// getri.cu -- inverse of a general matrix from its LU factors (getri, getri_outofplace and
// their npvt forms).
//
// Replaces library/src/lapack/roclapack_getri.hpp:265-390 (rocsolver_getri_template: trtri of
// U, then inv(A) L = inv(U) by blocked GEMM/TRSM, then column interchanges) and
// roclapack_getri_outofplace.hpp:73-127 (check_singularity, C = I, getrs on C).
//
// B200 design: orders whose member fits in 64 KB of shared memory (FP64 n <= 90, FP32
// n <= 128, complex double n <= 64, complex float n <= 90) are inverted on chip by one CTA
// per member with LAPACK's own unblocked steps (getri_small_kernel: one pass over the
// factors in, one over the inverse out).  Larger orders solve A C = I with the library's
// getrs kernels (one warp per matrix and right-hand-side group for n <= 32, otherwise one
// CTA per matrix and group of right-hand sides), after one prep kernel
// that finds the first zero diagonal entry of U (info, LAPACK dtrtri's singularity test) and
// writes the identity into C.  In-place getri solves into the handle workspace and copies
// the inverse back over the factors of the members with info = 0; members with info > 0 keep
// their factors (LAPACK dgetri returns before touching A), and for getri_outofplace their C
// holds the identity (the reference leaves it undefined).
#include "handle.h"
#include "launch.h"
#include "logger.h"

namespace rsb {

// 0, 1 and the zero test for the real and the complex element types
template <typename T>
struct GetriNum
{
    static constexpr bool complex_type = false;
    static __device__ T zero() { return T(0); }
    static __device__ T one() { return T(1); }
    static __device__ bool is_zero(T x) { return x == T(0); }
    static __device__ T add(T a, T b) { return a + b; }
    static __device__ T sub(T a, T b) { return a - b; }
    static __device__ T mul(T a, T b) { return a * b; }
    static __device__ T neg(T a) { return -a; }
    static __device__ T inv(T a) { return T(1) / a; }
};
template <typename C>
struct GetriNumC
{
    static constexpr bool complex_type = true;
    static __device__ C mk(double re, double im)
    {
        C z;
        z.x = re;
        z.y = im;
        return z;
    }
    static __device__ C zero() { return mk(0, 0); }
    static __device__ C one() { return mk(1, 0); }
    static __device__ bool is_zero(C x) { return x.x == 0 && x.y == 0; }
    static __device__ C add(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
    static __device__ C sub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
    static __device__ C mul(C a, C b) { return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
    static __device__ C neg(C a) { return mk(-a.x, -a.y); }
    // 1 / a by Smith's method (scaled by the larger component)
    static __device__ C inv(C a)
    {
        if(fabs(a.x) >= fabs(a.y))
        {
            const auto r = a.y / a.x, d = a.x + a.y * r;
            return mk(1 / d, -r / d);
        }
        const auto r = a.x / a.y, d = a.y + a.x * r;
        return mk(r / d, -1 / d);
    }
};
template <>
struct GetriNum<rocblas_float_complex> : GetriNumC<rocblas_float_complex>
{
};
template <>
struct GetriNum<rocblas_double_complex> : GetriNumC<rocblas_double_complex>
{
};

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
        if(GetriNum<T>::is_zero(a[ix(i, i, lda)]))
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
        w[ix(i, j, ldw)] = i == j ? GetriNum<T>::one() : GetriNum<T>::zero();
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

// ---- small orders: the whole inverse in shared memory, one CTA (one thread per row) per
// member, LAPACK's unblocked algorithm (dgetri = dtrti2 on U, then the solve of X L =
// inv(U) column by column from the right, then the column interchanges in reverse order).
// The member is read once and the inverse written once; no workspace.
constexpr int GETRI_SMALL_BYTES = 64 * 1024;

template <typename T>
static bool getri_small(int n)
{
    return n <= 128 && (size_t)n * n * sizeof(T) <= GETRI_SMALL_BYTES;
}

// C.base == C.ptrs == nullptr: the inverse overwrites A.  Members whose U has a zero diagonal
// entry get info = its order and keep A (getri_outofplace: C = I), as the prep kernel below.
template <typename T, int NT>
__global__ void __launch_bounds__(NT)
    getri_small_kernel(int n, Batch<T> A, int lda, const int* ipiv, int64_t strideP,
                       Batch<T> C, int ldc, int* info)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* s = reinterpret_cast<T*>(smem_raw); // n x n, leading dimension n
    __shared__ int first;
    const int64_t b = blockIdx.x;
    const int i = threadIdx.x; // this thread's row
    const T* a = A.at(b);
    const bool inplace = C.base == nullptr && C.ptrs == nullptr;
    T* out = inplace ? A.at(b) : C.at(b);
    const int ldo = inplace ? lda : ldc;
    if(i == 0)
        first = INT_MAX;
    __syncthreads();
    if(i < n)
    {
        for(int c = 0; c < n; ++c)
            s[i + c * n] = RSB_AT(a, i, c, lda, n, n);
        if(GetriNum<T>::is_zero(s[i + i * n]))
            atomicMin(&first, i);
    }
    __syncthreads();
    if(first != INT_MAX)
    {
        if(!inplace && i < n)
            for(int c = 0; c < n; ++c)
                RSB_AT(out, i, c, ldo, n, n) = i == c ? GetriNum<T>::one() : GetriNum<T>::zero();
        if(i == 0)
            info[b] = first + 1;
        return;
    }
    // inv(U) in place (dtrti2, upper, non-unit): column j = -inv(U)(j,j) * inv(U_11) U(0:j, j)
    for(int j = 0; j < n; ++j)
    {
        if(i == j)
            s[j + j * n] = GetriNum<T>::inv(s[j + j * n]);
        __syncthreads();
        T t = GetriNum<T>::zero();
        if(i < j)
            for(int k = i; k < j; ++k)
                t = GetriNum<T>::add(t, GetriNum<T>::mul(s[i + k * n], s[k + j * n]));
        const T ajj = GetriNum<T>::neg(s[j + j * n]);
        __syncthreads();
        if(i < j)
            s[i + j * n] = GetriNum<T>::mul(t, ajj);
    }
    __syncthreads();
    // X L = inv(U), columns from the right: X(:, j) -= X(:, j+1:n) L(j+1:n, j), L(:, j) -> 0
    for(int j = n - 2; j >= 0; --j)
    {
        T t = GetriNum<T>::zero();
        if(i < n)
            for(int k = j + 1; k < n; ++k)
                t = GetriNum<T>::add(t, GetriNum<T>::mul(s[i + k * n], s[k + j * n]));
        __syncthreads();
        if(i < n)
            s[i + j * n] = GetriNum<T>::sub(i > j ? GetriNum<T>::zero() : s[i + j * n], t);
        __syncthreads();
    }
    // column interchanges in reverse order, each thread on its own row
    if(i < n)
    {
        if(ipiv)
        {
            const int* piv = ipiv + b * strideP;
            for(int j = n - 2; j >= 0; --j)
            {
                const int jp = piv[j] - 1;
                RSB_CHECK_PIV(piv[j], n, __LINE__);
                if(jp != j && jp >= 0 && jp < n)
                {
                    const T tmp = s[i + j * n];
                    s[i + j * n] = s[i + jp * n];
                    s[i + jp * n] = tmp;
                }
            }
        }
        for(int c = 0; c < n; ++c)
            RSB_AT(out, i, c, ldo, n, n) = s[i + c * n];
    }
    if(i == 0)
        info[b] = 0;
}

template <typename T>
size_t getri_workspace(int n, int bc, bool inplace)
{
    return inplace && !getri_small<T>(n) ? ws_round(sizeof(T) * (size_t)n * n * bc) : 0;
}

template <typename T>
rocblas_status launch_getri(cudaStream_t s, int n, Batch<T> A, int lda, const int* ipiv,
                            int64_t strideP, Batch<T> C, int ldc, int* info, int bc, void* ws)
{
    if(getri_small<T>(n))
    {
        const size_t smem = sizeof(T) * (size_t)n * n;
        RSB_LOG_KERNEL("getri_small_kernel");
        if(n <= 64)
        {
            if(cudaFuncSetAttribute(getri_small_kernel<T, 64>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    GETRI_SMALL_BYTES)
               != cudaSuccess)
                return rocblas_status_internal_error;
            getri_small_kernel<T, 64><<<bc, 64, smem, s>>>(n, A, lda, ipiv, strideP, C, ldc, info);
        }
        else
        {
            if(cudaFuncSetAttribute(getri_small_kernel<T, 128>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    GETRI_SMALL_BYTES)
               != cudaSuccess)
                return rocblas_status_internal_error;
            getri_small_kernel<T, 128><<<bc, 128, smem, s>>>(n, A, lda, ipiv, strideP, C, ldc,
                                                             info);
        }
        return cudaGetLastError() == cudaSuccess ? rocblas_status_success
                                                 : rocblas_status_internal_error;
    }
    const bool inplace = C.base == nullptr && C.ptrs == nullptr;
    Batch<T> W = inplace ? strided<T>(static_cast<T*>(ws), (int64_t)n * n) : C;
    const int ldw = inplace ? n : ldc;
    {
        RSB_LOG_KERNEL("getri_prep_kernel");
        getri_prep_kernel<T><<<bc, 256, 0, s>>>(n, A, lda, W, ldw, info);
    }
    if(cudaGetLastError() != cudaSuccess)
        return rocblas_status_internal_error;
    rocblas_status st;
    if constexpr(GetriNum<T>::complex_type)
        st = launch_getrs<T>(s, 0, n, n, A, lda, ipiv, strideP, W, ldw, info, bc, no_gate());
    else
        st = launch_getrs_many<T>(s, n, n, A, lda, ipiv, strideP, W, ldw, info, bc);
    if(st != rocblas_status_success || !inplace)
        return st;
    RSB_LOG_KERNEL("getri_copy_back_kernel");
    getri_copy_back_kernel<T><<<bc, 256, 0, s>>>(n, W, ldw, A, lda, info);
    return cudaGetLastError() == cudaSuccess ? rocblas_status_success
                                             : rocblas_status_internal_error;
}

#define RSB_GETRI_INST(T)                                                                    \
    template size_t getri_workspace<T>(int, int, bool);                                      \
    template rocblas_status launch_getri<T>(cudaStream_t, int, Batch<T>, int, const int*,     \
                                            int64_t, Batch<T>, int, int*, int, void*);
RSB_GETRI_INST(float)
RSB_GETRI_INST(double)
RSB_GETRI_INST(rocblas_float_complex)
RSB_GETRI_INST(rocblas_double_complex)

} // namespace rsb
