// complex.cu -- the complex precisions (c = rocblas_float_complex, z = rocblas_double_complex)
// of the factor-and-solve path: getrf (and npvt), getrs (N, T, C), gesv, potrf, potrs, posv.
//
// The reference instantiates every hot-path routine for s, d, c and z
// (library/src/specialized/*_{s,d,c,z}.cpp); complex adds the conjugated solves
// (specialized/roclapack_trsm_specialized_kernels.hpp:219-380 conj_forward/backward
// substitution) and Hermitian Cholesky (roclapack_potf2.hpp:185-248 with conjugated dots).
//
// Design: one CTA of CPX_NT threads per matrix, working in place in global memory (members
// are L2-resident while their CTA runs).  getrf: per column a CTA-wide argmax of |re| + |im|
// (LAPACK izamax: first index of the maximum, a NaN only wins in the first position, through
// the same pivot keys as the real kernels), the row interchange over all columns, scaling by
// the reciprocal (|pivot| >= sfmin) or by division, and the rank-1 update of the trailing
// matrix spread over all threads (rows fastest: coalesced).  Solves sweep one unknown at a
// time with the updates of the remaining rows spread over the threads.  These kernels favour
// simplicity over speed: the tensor-core and register-resident kernels are FP32/FP64.
#include "handle.h"
#include "launch.h"
#include "logger.h"

namespace rsb {
namespace {

constexpr int CPX_NT = 256;

template <typename C>
struct CxReal;
template <>
struct CxReal<rocblas_float_complex>
{
    using R = float;
};
template <>
struct CxReal<rocblas_double_complex>
{
    using R = double;
};

template <typename C>
__device__ __forceinline__ C cx(typename CxReal<C>::R re, typename CxReal<C>::R im)
{
    C z;
    z.x = re;
    z.y = im;
    return z;
}
template <typename C>
__device__ __forceinline__ C cmul(C a, C b)
{
    return cx<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b)
{
    return cx<C>(a.x - b.x, a.y - b.y);
}
template <typename C>
__device__ __forceinline__ C cconj(C a)
{
    return cx<C>(a.x, -a.y);
}
template <typename C>
__device__ __forceinline__ bool czero(C a)
{
    return a.x == 0 && a.y == 0;
}
// a / b by Smith's method (scaled by the larger component of b)
template <typename C>
__device__ __forceinline__ C cdiv(C a, C b)
{
    using R = typename CxReal<C>::R;
    if(fabs(b.x) >= fabs(b.y))
    {
        const R r = b.y / b.x, d = b.x + b.y * r;
        return cx<C>((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    }
    const R r = b.x / b.y, d = b.y + b.x * r;
    return cx<C>((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}

// CTA-wide (key, row) argmax: largest key, smallest row on ties (LAPACK izamax order)
template <typename K>
__device__ int cta_argmax(K key, int row, bool valid, K* skey, int* srow)
{
    K wk;
    const int wr = warp_argmax(key, row, valid, &wk);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if(lane == 0)
    {
        skey[warp] = wk;
        srow[warp] = wr;
    }
    __syncthreads();
    const bool rv = lane < CPX_NT / 32 && srow[lane] != INT_MAX;
    K gk;
    const int gr = warp_argmax(rv ? skey[lane] : K(0), rv ? srow[lane] : INT_MAX, rv, &gk);
    __syncthreads();
    return gr;
}

template <typename C, bool PIVOT>
__global__ void __launch_bounds__(CPX_NT)
    cgetrf_kernel(int m, int n, Batch<C> A, int lda, int* ipiv, int64_t strideP, int* info,
                  Gate gate)
{
    using R = typename CxReal<C>::R;
    using K = typename KeyOf<R>::type;
    __shared__ K skey[CPX_NT / 32];
    __shared__ int srow[CPX_NT / 32];
    const int64_t b = blockIdx.x;
    if(gate.skip(b))
        return;
    C* a = A.at(b);
    const int tid = threadIdx.x;
    const int mn = min(m, n);
    int inf = 0;
    for(int j = 0; j < mn; ++j)
    {
        int p = j;
        if(PIVOT)
        {
            // this thread's first largest |re| + |im| among rows j + tid, j + tid + NT, ...
            K bk = 0;
            int br = INT_MAX;
            for(int i = j + tid; i < m; i += CPX_NT)
            {
                const C v = RSB_AT(a, i, j, lda, m, n);
                const K k = pivot_key((R)(fabs(v.x) + fabs(v.y)), i == j);
                if(br == INT_MAX || k > bk)
                {
                    bk = k;
                    br = i;
                }
            }
            p = cta_argmax(bk, br, br != INT_MAX, skey, srow);
            if(tid == 0)
                ipiv[b * strideP + j] = p + 1;
        }
        const C piv = RSB_AT(a, p, j, lda, m, n);
        __syncthreads();
        if(!czero(piv))
        {
            if(p != j)
                for(int c = tid; c < n; c += CPX_NT)
                {
                    const C t = RSB_AT(a, j, c, lda, m, n);
                    RSB_AT(a, j, c, lda, m, n) = RSB_AT(a, p, c, lda, m, n);
                    RSB_AT(a, p, c, lda, m, n) = t;
                }
            __syncthreads();
            const bool rec = hypot(piv.x, piv.y) >= Lim<R>::sfmin();
            const C r = rec ? cdiv(cx<C>(1, 0), piv) : piv;
            for(int i = j + 1 + tid; i < m; i += CPX_NT)
            {
                C& e = RSB_AT(a, i, j, lda, m, n);
                e = rec ? cmul(e, r) : cdiv(e, piv);
            }
        }
        else if(inf == 0)
            inf = j + 1;
        __syncthreads();
        // A(j+1:m, j+1:n) -= A(j+1:m, j) A(j, j+1:n)
        const int rows = m - j - 1, cols = n - j - 1;
        for(int64_t e = tid; e < (int64_t)rows * cols; e += CPX_NT)
        {
            const int i = j + 1 + (int)(e % rows), c = j + 1 + (int)(e / rows);
            const C u = RSB_AT(a, j, c, lda, m, n);
            if(!czero(u))
            {
                C& t = RSB_AT(a, i, c, lda, m, n);
                t = csub(t, cmul(RSB_AT(a, i, j, lda, m, n), u));
            }
        }
        __syncthreads();
    }
    if(tid == 0)
        info[b] = inf;
}

// B <- op(A)^{-1} B with the getrf factors: trans 0 = N, 1 = T, 2 = C (conjugate transpose).
template <typename C>
__global__ void __launch_bounds__(CPX_NT)
    cgetrs_kernel(int trans, int n, int nrhs, Batch<C> A, int lda, const int* ipiv,
                  int64_t strideP, Batch<C> B, int ldb, const int* skip, Gate gate)
{
    const int64_t b = blockIdx.x;
    if((skip && skip[b] != 0) || gate.skip(b))
        return;
    const C* a = A.at(b);
    C* x = B.at(b);
    const int* piv = ipiv ? ipiv + b * strideP : nullptr;
    const int tid = threadIdx.x;
    const bool cj = trans == 2;
    auto op = [&](int i, int j) {
        const C v = RSB_AT(a, i, j, lda, n, n);
        return cj ? cconj(v) : v;
    };
    auto swaps = [&](bool forward) {
        for(int c = tid; c < nrhs; c += CPX_NT)
            for(int s = 0; s < n; ++s)
            {
                const int k = forward ? s : n - 1 - s;
                const int p = piv[k] - 1;
                RSB_CHECK_PIV(piv[k], n, __LINE__);
                if(p != k)
                {
                    const C t = RSB_AT(x, k, c, ldb, n, nrhs);
                    RSB_AT(x, k, c, ldb, n, nrhs) = RSB_AT(x, p, c, ldb, n, nrhs);
                    RSB_AT(x, p, c, ldb, n, nrhs) = t;
                }
            }
        __syncthreads();
    };
    if(trans == 0)
    {
        if(piv)
            swaps(true);
        for(int k = 0; k < n; ++k) // L (unit lower)
        {
            for(int e = tid; e < (n - k - 1) * nrhs; e += CPX_NT)
            {
                const int i = k + 1 + e % (n - k - 1), c = e / (n - k - 1);
                C& t = RSB_AT(x, i, c, ldb, n, nrhs);
                t = csub(t, cmul(op(i, k), RSB_AT(x, k, c, ldb, n, nrhs)));
            }
            __syncthreads();
        }
        for(int k = n - 1; k >= 0; --k) // U
        {
            for(int c = tid; c < nrhs; c += CPX_NT)
                RSB_AT(x, k, c, ldb, n, nrhs) = cdiv(RSB_AT(x, k, c, ldb, n, nrhs), op(k, k));
            __syncthreads();
            for(int e = tid; e < k * nrhs; e += CPX_NT)
            {
                const int i = e % k, c = e / k;
                C& t = RSB_AT(x, i, c, ldb, n, nrhs);
                t = csub(t, cmul(op(i, k), RSB_AT(x, k, c, ldb, n, nrhs)));
            }
            __syncthreads();
        }
    }
    else
    {
        for(int k = 0; k < n; ++k) // op(U)^T: lower, entries op(U(k, i))
        {
            for(int c = tid; c < nrhs; c += CPX_NT)
                RSB_AT(x, k, c, ldb, n, nrhs) = cdiv(RSB_AT(x, k, c, ldb, n, nrhs), op(k, k));
            __syncthreads();
            for(int e = tid; e < (n - k - 1) * nrhs; e += CPX_NT)
            {
                const int i = k + 1 + e % (n - k - 1), c = e / (n - k - 1);
                C& t = RSB_AT(x, i, c, ldb, n, nrhs);
                t = csub(t, cmul(op(k, i), RSB_AT(x, k, c, ldb, n, nrhs)));
            }
            __syncthreads();
        }
        for(int k = n - 1; k >= 0; --k) // op(L)^T: unit upper, entries op(L(k, i))
        {
            for(int e = tid; e < k * nrhs; e += CPX_NT)
            {
                const int i = e % k, c = e / k;
                C& t = RSB_AT(x, i, c, ldb, n, nrhs);
                t = csub(t, cmul(op(k, i), RSB_AT(x, k, c, ldb, n, nrhs)));
            }
            __syncthreads();
        }
        if(piv)
            swaps(false);
    }
}

// Hermitian Cholesky, right-looking: A = L L^H (lower) or U^H U (upper); info = first order
// whose pivot real(a_jj) - sum |l_jk|^2 is <= 0 or NaN (that value is stored in a_jj, then
// the factorisation stops, as LAPACK zpotf2 does).  The other triangle is not touched.
template <typename C>
__global__ void __launch_bounds__(CPX_NT)
    cpotrf_kernel(int upper, int n, Batch<C> A, int lda, int* info)
{
    using R = typename CxReal<C>::R;
    const int64_t b = blockIdx.x;
    C* a = A.at(b);
    const int tid = threadIdx.x;
    for(int j = 0; j < n; ++j)
    {
        const R ajj = RSB_AT(a, j, j, lda, n, n).x;
        __syncthreads();
        if(ajj <= R(0) || isnan(ajj))
        {
            if(tid == 0)
            {
                RSB_AT(a, j, j, lda, n, n) = cx<C>(ajj, 0);
                info[b] = j + 1;
            }
            return;
        }
        const R d = sqrt(ajj), rd = R(1) / d;
        if(tid == 0)
            RSB_AT(a, j, j, lda, n, n) = cx<C>(d, 0);
        for(int i = j + 1 + tid; i < n; i += CPX_NT)
        {
            C& e = upper ? RSB_AT(a, j, i, lda, n, n) : RSB_AT(a, i, j, lda, n, n);
            e = cx<C>(e.x * rd, e.y * rd);
        }
        __syncthreads();
        // trailing Hermitian update of the referenced triangle
        const int t = n - j - 1;
        for(int64_t e = tid; e < (int64_t)t * t; e += CPX_NT)
        {
            const int i = j + 1 + (int)(e % t), k = j + 1 + (int)(e / t);
            if(!upper && i >= k) // L(i,k) -= L(i,j) conj(L(k,j))
            {
                C& v = RSB_AT(a, i, k, lda, n, n);
                v = csub(v, cmul(RSB_AT(a, i, j, lda, n, n), cconj(RSB_AT(a, k, j, lda, n, n))));
            }
            else if(upper && k >= i) // U(i,k) -= conj(U(j,i)) U(j,k)
            {
                C& v = RSB_AT(a, i, k, lda, n, n);
                v = csub(v, cmul(cconj(RSB_AT(a, j, i, lda, n, n)), RSB_AT(a, j, k, lda, n, n)));
            }
        }
        __syncthreads();
    }
    if(tid == 0)
        info[b] = 0;
}

// B <- A^{-1} B with the Cholesky factor: lower L Y = B, L^H X = Y; upper U^H Y = B, U X = Y.
template <typename C>
__global__ void __launch_bounds__(CPX_NT)
    cpotrs_kernel(int upper, int n, int nrhs, Batch<C> A, int lda, Batch<C> B, int ldb,
                  const int* skip)
{
    const int64_t b = blockIdx.x;
    if(skip && skip[b] != 0)
        return;
    const C* a = A.at(b);
    C* x = B.at(b);
    const int tid = threadIdx.x;
    // forward sweep with the lower factor M = L or U^H: M(i,k) for i > k
    auto mlo = [&](int i, int k) {
        return upper ? cconj(RSB_AT(a, k, i, lda, n, n)) : RSB_AT(a, i, k, lda, n, n);
    };
    for(int k = 0; k < n; ++k)
    {
        for(int c = tid; c < nrhs; c += CPX_NT)
            RSB_AT(x, k, c, ldb, n, nrhs) = cdiv(RSB_AT(x, k, c, ldb, n, nrhs), mlo(k, k));
        __syncthreads();
        for(int e = tid; e < (n - k - 1) * nrhs; e += CPX_NT)
        {
            const int i = k + 1 + e % (n - k - 1), c = e / (n - k - 1);
            C& t = RSB_AT(x, i, c, ldb, n, nrhs);
            t = csub(t, cmul(mlo(i, k), RSB_AT(x, k, c, ldb, n, nrhs)));
        }
        __syncthreads();
    }
    // backward sweep with M^H (upper): entries M^H(i,k) = conj(M(k,i)) for i < k
    for(int k = n - 1; k >= 0; --k)
    {
        for(int c = tid; c < nrhs; c += CPX_NT)
            RSB_AT(x, k, c, ldb, n, nrhs) =
                cdiv(RSB_AT(x, k, c, ldb, n, nrhs), cconj(mlo(k, k)));
        __syncthreads();
        for(int e = tid; e < k * nrhs; e += CPX_NT)
        {
            const int i = e % k, c = e / k;
            C& t = RSB_AT(x, i, c, ldb, n, nrhs);
            t = csub(t, cmul(cconj(mlo(k, i)), RSB_AT(x, k, c, ldb, n, nrhs)));
        }
        __syncthreads();
    }
}

inline rocblas_status status_of_launch()
{
    return cudaGetLastError() == cudaSuccess ? rocblas_status_success
                                             : rocblas_status_internal_error;
}

template <typename C>
rocblas_status cx_getrf(cudaStream_t s, int m, int n, Batch<C> A, int lda, int* ipiv,
                        int64_t sP, int* info, int bc, bool pivot, Gate g)
{
    RSB_LOG_KERNEL("cgetrf_kernel");
    if(pivot)
        cgetrf_kernel<C, true><<<bc, CPX_NT, 0, s>>>(m, n, A, lda, ipiv, sP, info, g);
    else
        cgetrf_kernel<C, false><<<bc, CPX_NT, 0, s>>>(m, n, A, lda, ipiv, sP, info, g);
    return status_of_launch();
}
template <typename C>
rocblas_status cx_getrs(cudaStream_t s, int trans, int n, int nrhs, Batch<C> A, int lda,
                        const int* ipiv, int64_t sP, Batch<C> B, int ldb, const int* skip,
                        int bc, Gate g)
{
    RSB_LOG_KERNEL("cgetrs_kernel");
    cgetrs_kernel<C><<<bc, CPX_NT, 0, s>>>(trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, g);
    return status_of_launch();
}
template <typename C>
rocblas_status cx_potrf(cudaStream_t s, int upper, int n, Batch<C> A, int lda, int* info, int bc)
{
    RSB_LOG_KERNEL("cpotrf_kernel");
    cpotrf_kernel<C><<<bc, CPX_NT, 0, s>>>(upper, n, A, lda, info);
    return status_of_launch();
}
template <typename C>
rocblas_status cx_potrs(cudaStream_t s, int upper, int n, int nrhs, Batch<C> A, int lda,
                        Batch<C> B, int ldb, const int* skip, int bc)
{
    RSB_LOG_KERNEL("cpotrs_kernel");
    cpotrs_kernel<C><<<bc, CPX_NT, 0, s>>>(upper, n, nrhs, A, lda, B, ldb, skip);
    return status_of_launch();
}

} // namespace

#define RSB_CPLX_LAUNCHERS(C)                                                                 \
    template <>                                                                               \
    rocblas_status launch_getrf<C>(cudaStream_t s, int m, int n, Batch<C> A, int lda,         \
                                   int* ipiv, int64_t sP, int* info, int bc, bool pivot,      \
                                   Gate g, bool)                                              \
    {                                                                                         \
        return cx_getrf<C>(s, m, n, A, lda, ipiv, sP, info, bc, pivot, g);                    \
    }                                                                                         \
    template <>                                                                               \
    rocblas_status launch_getrs<C>(cudaStream_t s, int trans, int n, int nrhs, Batch<C> A,    \
                                   int lda, const int* ipiv, int64_t sP, Batch<C> B, int ldb, \
                                   const int* skip, int bc, Gate g)                           \
    {                                                                                         \
        return cx_getrs<C>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc, g);         \
    }                                                                                         \
    template <>                                                                               \
    rocblas_status launch_gesv<C>(cudaStream_t s, int n, int nrhs, Batch<C> A, int lda,       \
                                  int* ipiv, int64_t sP, Batch<C> B, int ldb, int* info,      \
                                  int bc)                                                     \
    {                                                                                         \
        rocblas_status st = cx_getrf<C>(s, n, n, A, lda, ipiv, sP, info, bc, true, no_gate());\
        if(st != rocblas_status_success)                                                      \
            return st;                                                                        \
        return cx_getrs<C>(s, 0, n, nrhs, A, lda, ipiv, sP, B, ldb, info, bc, no_gate());     \
    }                                                                                         \
    template <>                                                                               \
    rocblas_status launch_potrf<C>(cudaStream_t s, int upper, int n, Batch<C> A, int lda,     \
                                   int* info, int bc)                                         \
    {                                                                                         \
        return cx_potrf<C>(s, upper, n, A, lda, info, bc);                                    \
    }                                                                                         \
    template <>                                                                               \
    rocblas_status launch_potrs<C>(cudaStream_t s, int upper, int n, int nrhs, Batch<C> A,    \
                                   int lda, Batch<C> B, int ldb, const int* skip, int bc)     \
    {                                                                                         \
        return cx_potrs<C>(s, upper, n, nrhs, A, lda, B, ldb, skip, bc);                      \
    }

RSB_CPLX_LAUNCHERS(rocblas_float_complex)
RSB_CPLX_LAUNCHERS(rocblas_double_complex)

} // namespace rsb
