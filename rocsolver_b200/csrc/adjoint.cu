// adjoint.cu -- adjoint (reverse-mode derivative) of the batched solve X = A^{-1} B.
//
// No counterpart in the reference.  Given the factors the forward solve already produced
// (getrf: P A = L U with ipiv; potrf: A = L L' or U' U) and the upstream gradient G = dL/dX:
//   gB = A^{-T} G          (getrs with trans = T: U' solve, L' solve, inverse row swaps,
//                           library/src/lapack/roclapack_getrs.hpp:134-150; for the SPD
//                           case gB = A^{-1} G with the Cholesky factor)
//   gA = -gB X^T           (rank-nrhs outer product)
// One CTA per matrix: the right-hand sides live in shared memory through both triangular
// sweeps, and gA is written straight from that shared-memory copy of gB, so the factors
// are read once and gA once written; no refactorisation and no workspace.
#include "launch.h"
#include "logger.h"
#include "trsv.cuh"

namespace rsb {

template <typename T, int NT, int NRC>
__global__ void __launch_bounds__(NT, 2)
    solve_adjoint_kernel(int kind, int n, int nrhs, Batch<T> A, int lda, const int* ipiv,
                         int64_t strideP, Batch<T> X, int ldx, Batch<T> G, int ldg, Batch<T> GA,
                         int ldga, Batch<T> GB, int ldgb)
{
    // kind: 0 = LU (getrf factors), 1 = Cholesky lower, 2 = Cholesky upper
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sdiag = reinterpret_cast<T*>(smem_raw); // staged diagonal blocks
    T* sg = sdiag + sweep_scratch<NT>();       // n x NRC  (gB columns of the group)
    T* sx = sg + (size_t)n * NRC;              // n x NRC  (X columns of the group)
    int* perm = reinterpret_cast<int*>(sx + (size_t)n * NRC);
    int* pinv = perm + n; // pinv[perm[i]] = i
    const int64_t b = blockIdx.x;
    const T* a = A.at(b);
    const T* x = X.at(b);
    const T* g = G.at(b);
    T* ga = GA.at(b);
    T* gb = GB.at(b);
    if(kind == 0)
    {
        build_perm(ipiv + b * strideP, n, perm);
        for(int i = threadIdx.x; i < n; i += NT)
            pinv[perm[i]] = i;
        __syncthreads();
    }
    for(int c0 = 0; c0 < nrhs; c0 += NRC)
    {
        const int nc = min(NRC, nrhs - c0);
        staged_copy<NT, 4>(
            n * NRC,
            [&](int e) {
                const int i = e % n, c = e / n;
                return c < nc ? g[ix(i, c0 + c, ldg)] : T(0);
            },
            [&](int e, T v) { sg[e] = v; });
        staged_copy<NT, 4>(
            n * NRC,
            [&](int e) {
                const int i = e % n, c = e / n;
                return c < nc ? x[ix(i, c0 + c, ldx)] : T(0);
            },
            [&](int e, T v) { sx[e] = v; });
        __syncthreads();
        if(kind == 0)
        {
            // A' y = g  with  A = P' L U  ->  U' L' (P y) = g
            block_sweep<T, NT, NRC, true>(false, TriView<T>{a, lda, 1}, n, sg, nc, sdiag);
            block_sweep<T, NT, NRC, false>(true, TriView<T>{a, lda, 1}, n, sg, nc, sdiag);
        }
        else if(kind == 1)
        {
            block_sweep<T, NT, NRC, true>(false, TriView<T>{a, 1, lda}, n, sg, nc, sdiag);
            block_sweep<T, NT, NRC, false>(false, TriView<T>{a, lda, 1}, n, sg, nc, sdiag);
        }
        else
        {
            block_sweep<T, NT, NRC, true>(false, TriView<T>{a, lda, 1}, n, sg, nc, sdiag);
            block_sweep<T, NT, NRC, false>(false, TriView<T>{a, 1, lda}, n, sg, nc, sdiag);
        }
        // gB (inverse row interchanges for LU: gB[perm[i]] = y[i], i.e. row r of gB is
        // y[pinv[r]]), stored along gB's rows
        for(int e = threadIdx.x; e < n * nc; e += NT)
        {
            const int r = e % n, c = e / n;
            const int src = kind == 0 ? pinv[r] : r;
            gb[ix(r, c0 + c, ldgb)] = sg[src + c * n];
        }
        // gA -= gB X' over this group: each thread keeps one row r of gB (its NRC values,
        // sg[pinv[r]] for LU since final row perm[i] holds sg[i]) in registers and walks
        // columns j; consecutive threads take consecutive rows (coalesced stores), and
        // when n <= NT the NT/n thread groups split the columns
        {
            const int P = n <= NT ? NT / n : 1;
            const int g = n <= NT ? (int)threadIdx.x / n : 0;
            const int rstep = n <= NT ? n : NT;
            for(int r = n <= NT ? (int)threadIdx.x % n : (int)threadIdx.x; r < n && g < P;
                r += rstep)
            {
                const int i = kind == 0 ? pinv[r] : r;
                T gr[NRC];
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                    gr[c] = c < nc ? sg[i + c * n] : T(0);
                for(int j = g; j < n; j += P)
                {
                    T acc = c0 == 0 ? T(0) : ga[ix(r, j, ldga)];
#pragma unroll
                    for(int c = 0; c < NRC; ++c)
                        acc = fma(-gr[c], sx[j + c * n], acc);
                    ga[ix(r, j, ldga)] = acc;
                }
                if(n <= NT)
                    break;
            }
        }
        __syncthreads();
    }
}

template <typename T>
rocblas_status launch_solve_adjoint(cudaStream_t s, int kind, int n, int nrhs, Batch<T> A,
                                    int lda, const int* ipiv, int64_t strideP, Batch<T> X,
                                    int ldx, Batch<T> G, int ldg, Batch<T> GA, int ldga,
                                    Batch<T> GB, int ldgb, int bc)
{
    constexpr int NT = 256;
    constexpr int NRC = 8;
    const size_t smem =
        sizeof(T) * (2 * (size_t)n * NRC + sweep_scratch<NT>()) + sizeof(int) * 2 * (size_t)n;
    if(smem > 200 * 1024)
        return rocblas_status_not_implemented;
    auto k = solve_adjoint_kernel<T, NT, NRC>;
    if(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
       != cudaSuccess)
        return rocblas_status_internal_error;
    RSB_LOG_KERNEL("solve_adjoint_kernel");
    k<<<bc, NT, smem, s>>>(kind, n, nrhs, A, lda, ipiv, strideP, X, ldx, G, ldg, GA, ldga, GB,
                           ldgb);
    return cudaGetLastError() == cudaSuccess ? rocblas_status_success
                                             : rocblas_status_internal_error;
}

template rocblas_status launch_solve_adjoint<float>(cudaStream_t, int, int, int, Batch<float>,
                                                    int, const int*, int64_t, Batch<float>, int,
                                                    Batch<float>, int, Batch<float>, int,
                                                    Batch<float>, int, int);
template rocblas_status launch_solve_adjoint<double>(cudaStream_t, int, int, int, Batch<double>,
                                                     int, const int*, int64_t, Batch<double>,
                                                     int, Batch<double>, int, Batch<double>, int,
                                                     Batch<double>, int, int);

} // namespace rsb
