// lu_small.cuh -- warp-per-matrix LU, triangular solve and fused gesv for m, n <= 32.
//
// Replaces the reference's getf2_small_kernel (specialized/roclapack_getf2_specialized_kernels.hpp:22-136,
// one thread per row with the pivot scanned serially by every thread through LDS and
// 3 barriers per column) and its substitution kernels for the small-n path
// (specialized/roclapack_trsm_specialized_kernels.hpp:167-623).
//
// B200 design: one 32-lane warp owns one matrix, lane i holds row i in registers.  The
// pivot search is a warp reduction with redux.sync (no shared-memory scan, no CTA
// barrier); the row interchange is a relabelling of the lanes (no data moves); the pivot
// row is broadcast through a double-buffered shared-memory row, ordered by __syncwarp.
// Four independent matrices share a 128-thread CTA.
#pragma once

#include "common.cuh"

namespace rsb {

constexpr int SMALL_WPB = 4; // matrices (warps) per CTA

// getrf for m <= 32, n <= NMAX (NMAX <= 32).  Writes LU, ipiv (1-based, PIVOT only)
// and info.
template <typename T, int NMAX, bool PIVOT>
__global__ void __launch_bounds__(32 * SMALL_WPB)
    getrf_warp_kernel(int m, int n, Batch<T> A, int lda, int* ipiv, int64_t strideP, int* info,
                      int bc, Gate gate)
{
    // pivot row, double-buffered; element NMAX holds the pivot's reciprocal.  Rows of
    // NMAX + 4 elements keep every row 16-byte aligned for the vector accesses.
    __shared__ __align__(16) T srow[SMALL_WPB][2][NMAX + 4];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t b = (int64_t)blockIdx.x * SMALL_WPB + warp;
    if(b >= bc || gate.skip(b))
        return;
    T* a = A.at(b);
    T r[NMAX];
#pragma unroll
    for(int j = 0; j < NMAX; ++j)
        r[j] = (lane < m && j < n) ? RSB_AT(a, lane, j, lda, m, n) : T(0);

    constexpr int VW = 16 / sizeof(T); // elements per 16-byte vector
    int myrow = lane;
    int mypiv = lane + 1;
    int inf = 0;
    const int mn = min(m, n);
#pragma unroll
    for(int k = 0; k < NMAX; ++k)
    {
        if(k < mn)
        {
            const int buf = k & 1;
            T* row = srow[warp][buf];
            // every lane forms its candidate's reciprocal while the reduction runs (off the
            // column's serial path); the winner publishes it
            const T rc = r[k] != T(0) ? Lim<T>::rcp(r[k]) : T(0);
            int prow = k;
            if(PIVOT)
                prow = warp_argmax_fast(pivot_key(r[k], myrow == k), myrow,
                                        lane < m && myrow >= k);
            if(myrow == prow)
            {
                // publish columns from the vector boundary at or below k (the extra leading
                // elements are never read) and the reciprocal of the pivot
#pragma unroll
                for(int j = 0; j < NMAX; j += VW)
                {
                    if(j + VW <= k)
                        continue;
                    if constexpr(sizeof(T) == 8)
                        *reinterpret_cast<double2*>(row + j) = make_double2(r[j], r[j + 1]);
                    else
                        *reinterpret_cast<float4*>(row + j) =
                            make_float4(r[j], r[j + 1], r[j + 2], r[j + 3]);
                }
                row[NMAX] = rc;
            }
            __syncwarp();
            const T piv = row[k];
            const T rcp = row[NMAX];
            if(lane == k)
                mypiv = prow + 1;
            if(piv == T(0) && inf == 0)
                inf = k + 1;
            if(PIVOT)
            {
                if(myrow == prow)
                    myrow = k;
                else if(myrow == k)
                    myrow = prow;
            }
            if(lane < m && myrow > k)
            {
                // LAPACK getf2 scaling: reciprocal when |pivot| >= sfmin, else division (a
                // branch uniform across the warp: the division only runs for a subnormal pivot)
                const T x = r[k];
                T l = x;
                if(fabs(piv) >= Lim<T>::sfmin())
                    l = x * rcp;
                else if(piv != T(0))
                    l = x / piv;
                r[k] = l;
#pragma unroll
                for(int j = 0; j < NMAX; j += VW)
                {
                    if(j + VW <= k)
                        continue;
                    T e[VW];
                    if constexpr(sizeof(T) == 8)
                    {
                        const double2 t = *reinterpret_cast<const double2*>(row + j);
                        e[0] = t.x;
                        e[1] = t.y;
                    }
                    else
                    {
                        const float4 t = *reinterpret_cast<const float4*>(row + j);
                        e[0] = t.x;
                        e[1] = t.y;
                        e[2] = t.z;
                        e[3] = t.w;
                    }
#pragma unroll
                    for(int u = 0; u < VW; ++u)
                        if(j + u > k)
                            r[j + u] = fma(-l, e[u], r[j + u]);
                }
            }
        }
    }
    if(lane < m)
    {
#pragma unroll
        for(int j = 0; j < NMAX; ++j)
            if(j < n)
                RSB_AT(a, myrow, j, lda, m, n) = r[j];
    }
    if(PIVOT && lane < mn)
        ipiv[b * strideP + lane] = mypiv;
    if(lane == 0)
        info[b] = inf;
}

// Source-row map of the row interchanges ipiv[0..n-1]: after applying the swaps in order
// (LAPACK dlaswp, incx = 1) position i holds original row src (returned for lane i).
// Interchange k maps a'[i] = a[f_k(i)] with f_k the transposition (k, ipiv[k]-1), so
// src(i) = f_0(f_1(...f_{n-1}(i))): each lane composes the transpositions for its own
// position, one broadcast pivot per step (no serial chain of dependent shuffles).
__device__ __forceinline__ int warp_perm_src(const int* piv, int n, int lane)
{
    const unsigned full = 0xffffffffu;
    if(lane < n)
        RSB_CHECK_PIV(piv[lane], n, __LINE__);
    const int pv = lane < n ? piv[lane] - 1 : lane;
    int x = lane;
    for(int k = n - 1; k >= 0; --k)
    {
        const int p = __shfl_sync(full, pv, k);
        x = x == k ? p : (x == p ? k : x);
    }
    return (x >= 0 && x < n) ? x : lane;
}

// getrs for n <= NMAX <= 32 (library/src/lapack/roclapack_getrs.hpp:117-150 order:
// laswp, L (unit), U; or U', L' (unit), laswp backwards).  One warp per (matrix, group
// of NRC right-hand sides).  trans == 0: lane i holds row i of LU; trans != 0: lane i
// holds column i, so that both sweeps only need shuffles of the solved unknown.
template <typename T, int NMAX, int NRC>
__global__ void __launch_bounds__(32 * SMALL_WPB)
    getrs_warp_kernel(int trans, int n, int nrhs, Batch<T> A, int lda, const int* ipiv,
                      int64_t strideP, Batch<T> B, int ldb, const int* skip_info, int bc,
                      Gate gate)
{
    const unsigned full = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int groups = (nrhs + NRC - 1) / NRC;
    const int64_t task = (int64_t)blockIdx.x * SMALL_WPB + warp;
    if(task >= (int64_t)bc * groups)
        return;
    const int64_t b = task / groups;
    const int c0 = (int)(task % groups) * NRC;
    if((skip_info && skip_info[b] != 0) || gate.skip(b))
        return;
    const T* a = A.at(b);
    T* x = B.at(b);
    T r[NMAX];
#pragma unroll
    for(int j = 0; j < NMAX; ++j)
        r[j] = (lane < n && j < n) ? (trans ? RSB_AT(a, j, lane, lda, n, n)
                                           : RSB_AT(a, lane, j, lda, n, n))
                                   : T(0);
    const int src = ipiv ? warp_perm_src(ipiv + b * strideP, n, lane) : lane;
    // reciprocal of this lane's diagonal entry U(lane, lane), computed off the sweeps'
    // serial path (the sweeps multiply by it, as the reference's trsm applies inverted
    // diagonal blocks)
    T diag = T(1);
#pragma unroll
    for(int j = 0; j < NMAX; ++j)
        if(j == lane)
            diag = r[j];
    const T rdiag = T(1) / diag;

    T v[NRC];
#pragma unroll
    for(int c = 0; c < NRC; ++c)
        v[c] = (lane < n && c0 + c < nrhs) ? RSB_AT(x, trans ? lane : src, c0 + c, ldb, n, nrhs)
                                           : T(0);

    if(!trans)
    {
        // L y = P b (unit lower, column-oriented as reference dtrsm)
#pragma unroll
        for(int k = 0; k < NMAX; ++k)
        {
            if(k < n)
            {
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                {
                    T yk = __shfl_sync(full, v[c], k);
                    if(lane > k)
                        v[c] = fma(-r[k], yk, v[c]);
                }
            }
        }
        // U x = y
#pragma unroll
        for(int k = NMAX - 1; k >= 0; --k)
        {
            if(k < n)
            {
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                {
                    if(lane == k)
                        v[c] = v[c] * rdiag;
                    T xk = __shfl_sync(full, v[c], k);
                    if(lane < k)
                        v[c] = fma(-r[k], xk, v[c]);
                }
            }
        }
    }
    else
    {
        // U' y = b: lane i holds column i of U, so (U')(i,k) = U(k,i) = r[k] on lane i
#pragma unroll
        for(int k = 0; k < NMAX; ++k)
        {
            if(k < n)
            {
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                {
                    if(lane == k)
                        v[c] = v[c] * rdiag;
                    T yk = __shfl_sync(full, v[c], k);
                    if(lane > k)
                        v[c] = fma(-r[k], yk, v[c]);
                }
            }
        }
        // L' x = y (unit)
#pragma unroll
        for(int k = NMAX - 1; k >= 0; --k)
        {
            if(k < n)
            {
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                {
                    T xk = __shfl_sync(full, v[c], k);
                    if(lane < k)
                        v[c] = fma(-r[k], xk, v[c]);
                }
            }
        }
    }
    __syncwarp();
#pragma unroll
    for(int c = 0; c < NRC; ++c)
        if(lane < n && c0 + c < nrhs)
            RSB_AT(x, trans ? src : lane, c0 + c, ldb, n, nrhs) = v[c];
}

// Fused gesv for n <= NMAX <= 32 on one warp: factor in registers, then solve with the
// factors still in registers (no re-read of LU).  B is written only where info == 0,
// which is the reference's contract (library/src/lapack/roclapack_gesv.hpp:163-176
// restores B for failed members).  srow: [2][NMAX] and sown: [32] of this warp.
template <typename T, int NMAX, int NRC>
__device__ __forceinline__ void gesv_warp_dev(int n, int nrhs, T* a, int lda, int* piv, T* x,
                                              int ldb, int* info_out, T (*srow)[NMAX],
                                              int* sown)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    T r[NMAX];
#pragma unroll
    for(int j = 0; j < NMAX; ++j)
        r[j] = (lane < n && j < n) ? a[ix(lane, j, lda)] : T(0);
    int myrow = lane;
    int mypiv = lane + 1;
    int inf = 0;
#pragma unroll
    for(int k = 0; k < NMAX; ++k)
    {
        if(k < n)
        {
            const int buf = k & 1;
            // every lane forms the reciprocal of its candidate while the reductions run
            const T rck = r[k] != T(0) ? Lim<T>::rcp(r[k]) : T(0);
            typename KeyOf<T>::type kk;
            const int prow = warp_argmax(pivot_key(r[k], myrow == k), myrow,
                                         lane < n && myrow >= k, &kk);
            if(myrow == prow)
            {
#pragma unroll
                for(int j = k; j < NMAX; ++j)
                    srow[buf][j] = r[j];
            }
            const int wl = __ffs(__ballot_sync(full, myrow == prow)) - 1;
            const T rcp = __shfl_sync(full, rck, wl < 0 ? 0 : wl);
            __syncwarp();
            const T pivv = srow[buf][k];
            if(lane == k)
                mypiv = prow + 1;
            if(pivv == T(0) && inf == 0)
                inf = k + 1;
            if(myrow == prow)
                myrow = k;
            else if(myrow == k)
                myrow = prow;
            if(lane < n && myrow > k)
            {
                const T l = getf2_scale(r[k], pivv, rcp);
                r[k] = l;
#pragma unroll
                for(int j = k + 1; j < NMAX; ++j)
                    r[j] = fma(-l, srow[buf][j], r[j]);
            }
        }
    }
    if(lane < n)
    {
#pragma unroll
        for(int j = 0; j < NMAX; ++j)
            if(j < n)
                a[ix(myrow, j, lda)] = r[j];
        piv[lane] = mypiv;
        sown[myrow] = lane;
    }
    if(lane == 0)
        *info_out = inf;
    if(inf != 0)
        return; // uniform: B stays untouched
    __syncwarp();
    // reciprocal of this lane's diagonal entry U(myrow, myrow), off the serial path
    T diag = T(1);
#pragma unroll
    for(int j = 0; j < NMAX; ++j)
        if(j == myrow)
            diag = r[j];
    const T rdiag = T(1) / diag;
    for(int c0 = 0; c0 < nrhs; c0 += NRC)
    {
        // lane holds original row `lane` of B, which is position myrow of P*B
        T v[NRC];
#pragma unroll
        for(int c = 0; c < NRC; ++c)
            v[c] = (lane < n && c0 + c < nrhs) ? x[ix(lane, c0 + c, ldb)] : T(0);
#pragma unroll
        for(int k = 0; k < NMAX; ++k)
        {
            if(k < n)
            {
                const int o = sown[k];
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                {
                    T yk = __shfl_sync(full, v[c], o);
                    if(lane < n && myrow > k)
                        v[c] = fma(-r[k], yk, v[c]);
                }
            }
        }
#pragma unroll
        for(int k = NMAX - 1; k >= 0; --k)
        {
            if(k < n)
            {
                const int o = sown[k];
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                {
                    if(lane == o)
                        v[c] = v[c] * rdiag;
                    T xk = __shfl_sync(full, v[c], o);
                    if(lane < n && myrow < k)
                        v[c] = fma(-r[k], xk, v[c]);
                }
            }
        }
        __syncwarp();
#pragma unroll
        for(int c = 0; c < NRC; ++c)
            if(lane < n && c0 + c < nrhs)
                x[ix(myrow, c0 + c, ldb)] = v[c];
        __syncwarp();
    }
}

template <typename T, int NMAX, int NRC>
__global__ void __launch_bounds__(32 * SMALL_WPB)
    gesv_warp_kernel(int n, int nrhs, Batch<T> A, int lda, int* ipiv, int64_t strideP,
                     Batch<T> B, int ldb, int* info, int bc)
{
    __shared__ T srow[SMALL_WPB][2][NMAX];
    __shared__ int sown[SMALL_WPB][32];
    const int warp = threadIdx.x >> 5;
    const int64_t b = (int64_t)blockIdx.x * SMALL_WPB + warp;
    if(b >= bc)
        return;
    gesv_warp_dev<T, NMAX, NRC>(n, nrhs, A.at(b), lda, ipiv + b * strideP, B.at(b), ldb, info + b,
                                srow[warp], sown[warp]);
}

} // namespace rsb
