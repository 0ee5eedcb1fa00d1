// trsv.cuh -- CTA-per-matrix blocked triangular solves with several right-hand sides,
// used by getrs (n > 32), potrs and the solve adjoint.
//
// Replaces the reference's rocsolver_trsm_lower/upper drivers
// (specialized/roclapack_trsm_specialized_kernels.hpp:755-997, 1007-1249: a substitution
// kernel per diagonal block plus a rocBLAS GEMM per off-diagonal block, several launches
// per sweep) and laswp (auxiliary/rocauxiliary_laswp.hpp:18-64).
//
// One CTA per (matrix, group of NRC right-hand sides); the right-hand sides live in
// shared memory for the whole solve.  A sweep walks 32-wide diagonal blocks: warp 0
// solves the block with shuffles (no barrier), then all threads apply the block to the
// remaining rows (a GEMV reading the factor once, coalesced along its columns).
// A triangular operand is addressed as M(r, c) = base[r*rs + c*cs], so transposes are
// a swap of (rs, cs).
#pragma once

#include "common.cuh"

namespace rsb {

template <typename T>
struct TriView
{
    const T* p;
    int64_t rs, cs;
    __device__ __forceinline__ T operator()(int r, int c) const
    {
        return p[(int64_t)r * rs + (int64_t)c * cs];
    }
};

constexpr int SDIAG_LD = 33;               // staged diagonal block, padded
constexpr int SDIAG_ELEMS = 32 * SDIAG_LD;

// Solve M x = b in place for the nc columns of sb (ld = n).  forward: M lower
// (substitution top-down), else M upper (bottom-up).  unit: unit diagonal.
// sdiag: shared scratch of SDIAG_ELEMS elements.  Must be called by all NT threads.
// Per 32-wide block: all threads stage the diagonal block in shared memory (coalesced
// along the operand's contiguous direction), warp 0 solves it with shuffles, then all
// threads apply it to the remaining rows with independent (unrolled) factor loads.
template <typename T, int NT, int NRC>
__device__ void block_sweep(bool forward, bool unit, TriView<T> M, int n, T* sb, int nc,
                            T* sdiag)
{
    const unsigned full = 0xffffffffu;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nblk = (n + 31) / 32;
    for(int bi = 0; bi < nblk; ++bi)
    {
        const int kb = forward ? bi * 32 : (nblk - 1 - bi) * 32;
        const int nb = min(32, n - kb);
        for(int e = tid; e < nb * nb; e += NT)
        {
            int r, c;
            if(M.rs == 1)
            {
                r = e % nb;
                c = e / nb;
            }
            else
            {
                c = e % nb;
                r = e / nb;
            }
            sdiag[c * SDIAG_LD + r] = M(kb + r, kb + c);
        }
        __syncthreads();
        if(warp == 0)
        {
            T x[NRC];
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                x[c] = (lane < nb && c < nc) ? sb[kb + lane + c * n] : T(0);
            if(forward)
            {
                for(int k = 0; k < nb; ++k)
                {
                    const T mlk = sdiag[k * SDIAG_LD + lane];
                    const T dkk = unit ? T(1) : sdiag[k * SDIAG_LD + k];
#pragma unroll
                    for(int c = 0; c < NRC; ++c)
                    {
                        if(!unit && lane == k)
                            x[c] = x[c] / dkk;
                        const T xk = __shfl_sync(full, x[c], k);
                        if(lane > k && lane < nb)
                            x[c] = fma(-mlk, xk, x[c]);
                    }
                }
            }
            else
            {
                for(int k = nb - 1; k >= 0; --k)
                {
                    const T mlk = sdiag[k * SDIAG_LD + lane];
                    const T dkk = unit ? T(1) : sdiag[k * SDIAG_LD + k];
#pragma unroll
                    for(int c = 0; c < NRC; ++c)
                    {
                        if(!unit && lane == k)
                            x[c] = x[c] / dkk;
                        const T xk = __shfl_sync(full, x[c], k);
                        if(lane < k)
                            x[c] = fma(-mlk, xk, x[c]);
                    }
                }
            }
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                if(lane < nb && c < nc)
                    sb[kb + lane + c * n] = x[c];
        }
        __syncthreads();
        // rows outside the block: forward -> below it, backward -> above it
        const int r0 = forward ? kb + nb : 0;
        const int r1 = forward ? n : kb;
        for(int i = r0 + tid; i < r1; i += NT)
        {
            T acc[NRC];
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                acc[c] = c < nc ? sb[i + c * n] : T(0);
            if(nb == 32)
            {
                T mv[32];
#pragma unroll
                for(int k = 0; k < 32; ++k)
                    mv[k] = M(i, kb + k);
#pragma unroll
                for(int k = 0; k < 32; ++k)
#pragma unroll
                    for(int c = 0; c < NRC; ++c)
                        acc[c] = fma(-mv[k], sb[kb + k + c * n], acc[c]);
            }
            else
            {
                for(int k = 0; k < nb; ++k)
                {
                    const T mik = M(i, kb + k);
#pragma unroll
                    for(int c = 0; c < NRC; ++c)
                        acc[c] = fma(-mik, sb[kb + k + c * n], acc[c]);
                }
            }
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                if(c < nc)
                    sb[i + c * n] = acc[c];
        }
        __syncthreads();
    }
}

// Source map of LAPACK dlaswp(k1=1, k2=n, incx=1): position i receives original row
// perm[i].  Applying interchange k to an array maps a'[i] = a[f_k(i)] with f_k the
// transposition (k, piv[k]-1), so after all n interchanges perm[i] = f_0(f_1(...f_{n-1}(i))).
// For n <= 2*blockDim.x every thread evaluates that composition for its own positions
// (k from n-1 down to 0, pivots staged in shared memory and read as broadcasts): no
// serial chain through memory.
// Larger n replays the interchanges serially in one thread.  A pivot outside [1, n] never
// yields an index outside the matrix.
__device__ __forceinline__ void build_perm(const int* piv, int n, int* perm)
{
    const int nt = blockDim.x;
    if(n <= 2 * nt)
    {
        // pivots staged in perm[] (one coalesced load), read back as broadcasts
        for(int k = threadIdx.x; k < n; k += nt)
            perm[k] = piv[k] - 1;
        __syncthreads();
        const int i0 = threadIdx.x, i1 = threadIdx.x + nt;
        int x0 = i0, x1 = i1;
        int k = n - 1;
        for(; k >= 7; k -= 8)
        {
            int p[8];
#pragma unroll
            for(int u = 0; u < 8; ++u)
                p[u] = perm[k - u];
#pragma unroll
            for(int u = 0; u < 8; ++u)
            {
                const int kk = k - u;
                x0 = x0 == kk ? p[u] : (x0 == p[u] ? kk : x0);
                x1 = x1 == kk ? p[u] : (x1 == p[u] ? kk : x1);
            }
        }
        for(; k >= 0; --k)
        {
            const int p = perm[k];
            x0 = x0 == k ? p : (x0 == p ? k : x0);
            x1 = x1 == k ? p : (x1 == p ? k : x1);
        }
        __syncthreads();
        // an out-of-range pivot can only have produced an out-of-range x: keep the row
        if(i0 < n)
            perm[i0] = (x0 >= 0 && x0 < n) ? x0 : i0;
        if(i1 < n)
            perm[i1] = (x1 >= 0 && x1 < n) ? x1 : i1;
        __syncthreads();
        return;
    }
    for(int i = threadIdx.x; i < n; i += nt)
        perm[i] = i;
    __syncthreads();
    if(threadIdx.x == 0)
    {
        for(int k = 0; k < n; ++k)
        {
            const int p = piv[k] - 1;
            if(p != k && p >= 0 && p < n)
            {
                const int t = perm[k];
                perm[k] = perm[p];
                perm[p] = t;
            }
        }
    }
    __syncthreads();
}

// Solve with getrf factors for all nrhs columns (groups of NRC through shared memory
// sb[n*NRC] and perm[n]).  Called by all threads of the CTA.
template <typename T, int NT, int NRC>
__device__ __forceinline__ void getrs_dev(int trans, int n, int nrhs, const T* a, int lda,
                                          const int* piv, T* x, int ldb, T* sb, int* perm,
                                          T* sdiag)
{
    if(piv)
        build_perm(piv, n, perm);
    for(int c0 = 0; c0 < nrhs; c0 += NRC)
    {
        const int nc = min(NRC, nrhs - c0);
        for(int e = threadIdx.x; e < n * nc; e += NT)
        {
            const int i = e % n, c = e / n;
            const int src = (!trans && piv) ? perm[i] : i;
            sb[i + c * n] = x[ix(src, c0 + c, ldb)];
        }
        __syncthreads();
        if(!trans)
        {
            block_sweep<T, NT, NRC>(true, true, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
            block_sweep<T, NT, NRC>(false, false, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
        }
        else
        {
            block_sweep<T, NT, NRC>(true, false, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
            block_sweep<T, NT, NRC>(false, true, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
        }
        for(int e = threadIdx.x; e < n * nc; e += NT)
        {
            const int i = e % n, c = e / n;
            const int dst = (trans && piv) ? perm[i] : i;
            x[ix(dst, c0 + c, ldb)] = sb[i + c * n];
        }
        __syncthreads();
    }
}

// getrs for any n: trans == 0: P b, L (unit) forward, U backward;
// trans != 0: U' forward, L' (unit) backward, P' x.
// (library/src/lapack/roclapack_getrs.hpp:117-150)
template <typename T, int NT, int NRC>
__global__ void __launch_bounds__(NT, NT <= 128 ? 1024 / NT : 2)
    getrs_cta_kernel(int trans, int n, int nrhs, Batch<T> A, int lda, const int* ipiv,
                     int64_t strideP, Batch<T> B, int ldb, const int* skip_info, Gate gate)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sdiag = reinterpret_cast<T*>(smem_raw);
    T* sb = sdiag + SDIAG_ELEMS;
    int* perm = reinterpret_cast<int*>(sb + (size_t)n * NRC);
    const int groups = (nrhs + NRC - 1) / NRC;
    const int64_t b = blockIdx.x / groups;
    const int c0 = (blockIdx.x % groups) * NRC;
    const int nc = min(NRC, nrhs - c0);
    if((skip_info && skip_info[b] != 0) || gate.skip(b))
        return;
    const T* a = A.at(b);
    T* x = B.at(b);
    const bool pv = ipiv != nullptr;
    if(pv)
        build_perm(ipiv + b * strideP, n, perm);
    for(int e = threadIdx.x; e < n * nc; e += NT)
    {
        const int i = e % n, c = e / n;
        const int src = (!trans && pv) ? perm[i] : i;
        sb[i + c * n] = x[ix(src, c0 + c, ldb)];
    }
    __syncthreads();
    if(!trans)
    {
        block_sweep<T, NT, NRC>(true, true, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
        block_sweep<T, NT, NRC>(false, false, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
    }
    else
    {
        block_sweep<T, NT, NRC>(true, false, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
        block_sweep<T, NT, NRC>(false, true, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
    }
    for(int e = threadIdx.x; e < n * nc; e += NT)
    {
        const int i = e % n, c = e / n;
        const int dst = (trans && pv) ? perm[i] : i;
        x[ix(dst, c0 + c, ldb)] = sb[i + c * n];
    }
}

// potrs for any n: A = L L' (lower) or U' U (upper)
// (library/src/lapack/roclapack_potrs.hpp:87-152).
template <typename T, int NT, int NRC>
__global__ void __launch_bounds__(NT, NT <= 128 ? 1024 / NT : 2)
    potrs_cta_kernel(int upper, int n, int nrhs, Batch<T> A, int lda, Batch<T> B, int ldb,
                     const int* skip_info)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sdiag = reinterpret_cast<T*>(smem_raw);
    T* sb = sdiag + SDIAG_ELEMS;
    const int groups = (nrhs + NRC - 1) / NRC;
    const int64_t b = blockIdx.x / groups;
    const int c0 = (blockIdx.x % groups) * NRC;
    const int nc = min(NRC, nrhs - c0);
    if(skip_info && skip_info[b] != 0)
        return;
    const T* a = A.at(b);
    T* x = B.at(b);
    for(int e = threadIdx.x; e < n * nc; e += NT)
    {
        const int i = e % n, c = e / n;
        sb[i + c * n] = x[ix(i, c0 + c, ldb)];
    }
    __syncthreads();
    if(!upper)
    {
        block_sweep<T, NT, NRC>(true, false, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
        block_sweep<T, NT, NRC>(false, false, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
    }
    else
    {
        block_sweep<T, NT, NRC>(true, false, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
        block_sweep<T, NT, NRC>(false, false, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
    }
    for(int e = threadIdx.x; e < n * nc; e += NT)
    {
        const int i = e % n, c = e / n;
        x[ix(i, c0 + c, ldb)] = sb[i + c * n];
    }
}

// potrs for n <= N (N = 32 or 64 threads, one row each): the factor's triangle is staged
// in shared memory once (coalesced along its stored direction), each thread keeps its
// row's NRC right-hand-side values in registers, and both sweeps take one barrier per
// column: the row owning column c finalises its value (times the reciprocal of the
// diagonal, computed once per row off the critical path) and publishes it in a
// double-buffered slot; the rows still to be solved subtract their multiple of it.
template <typename T, int N, int NRC>
__global__ void __launch_bounds__(N, N <= 32 ? 16 : 8)
    potrs_small_kernel(int upper, int n, int nrhs, Batch<T> A, int lda, Batch<T> B, int ldb,
                       const int* skip_info)
{
    constexpr int LD = N + 1;
    __shared__ T sL[N * LD]; // L(r, c) at sL[r + c*LD], lower triangle
    __shared__ T sx[2][NRC];
    const int r = threadIdx.x;
    const int groups = (nrhs + NRC - 1) / NRC;
    const int64_t b = blockIdx.x / groups;
    const int c0 = (blockIdx.x % groups) * NRC;
    const int nc = min(NRC, nrhs - c0);
    if(skip_info && skip_info[b] != 0)
        return;
    const T* a = A.at(b);
    T* x = B.at(b);
    // L(i, j) = a[i + j*lda] (lower) or U(j, i) = a[j + i*lda] (upper); the fastest thread
    // index runs along the stored column either way
    for(int e = r; e < N * N; e += N)
    {
        const int p = e % N, q = e / N;
        const int i = upper ? q : p, j = upper ? p : q; // L(i, j), i >= j
        if(i < n && j <= i)
            sL[i + j * LD] = upper ? a[ix(j, i, lda)] : a[ix(i, j, lda)];
    }
    T v[NRC];
#pragma unroll
    for(int k = 0; k < NRC; ++k)
        v[k] = (r < n && k < nc) ? x[ix(r, c0 + k, ldb)] : T(0);
    __syncthreads();
    const T rd = r < n ? T(1) / sL[r + r * LD] : T(0);
    // forward: L y = b
#pragma unroll 1
    for(int c = 0; c < n; ++c)
    {
        const int buf = c & 1;
        if(r == c)
        {
#pragma unroll
            for(int k = 0; k < NRC; ++k)
            {
                v[k] *= rd;
                sx[buf][k] = v[k];
            }
        }
        __syncthreads();
        if(r > c && r < n)
        {
            const T l = sL[r + c * LD];
#pragma unroll
            for(int k = 0; k < NRC; ++k)
                v[k] = fma(-l, sx[buf][k], v[k]);
        }
    }
    // backward: L' x = y
#pragma unroll 1
    for(int c = n - 1; c >= 0; --c)
    {
        const int buf = (c + 1) & 1; // step n-1 takes the buffer the forward sweep did not end on
        if(r == c)
        {
#pragma unroll
            for(int k = 0; k < NRC; ++k)
            {
                v[k] *= rd;
                sx[buf][k] = v[k];
            }
        }
        __syncthreads();
        if(r < c)
        {
            const T l = sL[c + r * LD];
#pragma unroll
            for(int k = 0; k < NRC; ++k)
                v[k] = fma(-l, sx[buf][k], v[k]);
        }
    }
    if(r < n)
    {
#pragma unroll
        for(int k = 0; k < NRC; ++k)
            if(k < nc)
                x[ix(r, c0 + k, ldb)] = v[k];
    }
}

} // namespace rsb
