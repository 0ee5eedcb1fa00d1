// chol.cuh -- CTA-per-matrix blocked Cholesky for general n (lower or upper).
//
// Replaces the reference's potrf (library/src/lapack/roclapack_potrf.hpp:90-228) and its
// unblocked potf2 (library/src/lapack/roclapack_potf2.hpp:137-253), which at n = 64 issues
// ~256 launches per call (dot, sqrtDiagOnward with 1-thread blocks, gemv, scal per column).
//
// B200 design: ONE launch, one CTA per matrix.  The panel (rows j0..n-1 of JB columns of
// the referenced triangle) is held in registers, one or more rows per thread.  Per column
// the rows of the diagonal block publish their current column value to shared memory and
// one barrier later every thread has the pivot and the column of L it needs for its own
// rank-1 update.  For n <= JB (e.g. n = 64) the whole factorisation is one panel.  Wider
// matrices apply the panel to the trailing triangle (SYRK) with the L21 rows still in
// registers and the transposed operand broadcast from shared memory.
//
// The upper case (A = U' U) is the lower algorithm on the transposed view
// M(r, c) = A[c + r*lda].  The first non-positive (or NaN) pivot is stored, info is set to
// its 1-based index and the factorisation stops, as LAPACK dpotf2 does; the reference
// (sqrtDiagOnward, :16-43) records the same info.
#pragma once

#include "common.cuh"

namespace rsb {

template <typename T, int NT, int R, int JB>
struct CtaCholSmem
{
    static __host__ __device__ size_t bytes(int n)
    {
        (void)n;
        size_t s = sizeof(T) * 2 * JB + sizeof(T) * (size_t)R * NT * (JB + 1);
        return (s + 15) & ~size_t(15);
    }
};

template <typename T, int NT, int R, int JB, int TN>
__global__ void __launch_bounds__(NT)
    potrf_cta_kernel(int upper, int n, Batch<T> A, int lda, int* info)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* scol = reinterpret_cast<T*>(smem_raw);      // [2][JB]
    T* sL = scol + 2 * JB;                           // [R*NT][JB+1] trailing L rows
    constexpr int LDL = JB + 1;
    const int tid = threadIdx.x;
    const int64_t b = blockIdx.x;
    T* a = A.at(b);
    const int64_t rs = upper ? lda : 1, cs = upper ? 1 : lda;
    auto at = [&](int r, int c) -> T& { return a[(int64_t)r * rs + (int64_t)c * cs]; };

    T pv[R][JB];
    int inf = 0;
    for(int j0 = 0; j0 < n && inf == 0; j0 += JB)
    {
        const int jb = min(JB, n - j0);
        const int mp = n - j0;
#pragma unroll
        for(int q = 0; q < R; ++q)
        {
            const int r = tid + q * NT;
#pragma unroll
            for(int c = 0; c < JB; ++c)
                pv[q][c] = (r < mp && c < jb && c <= r) ? at(j0 + r, j0 + c) : T(0);
        }
        int cfail = JB;
#pragma unroll
        for(int c = 0; c < JB; ++c)
        {
            if(c < jb && cfail == JB)
            {
                const int buf = c & 1;
                T* sc = scol + buf * JB;
#pragma unroll
                for(int q = 0; q < R; ++q)
                {
                    const int r = tid + q * NT;
                    if(r >= c && r < jb)
                        sc[r] = pv[q][c];
                }
                __syncthreads();
                const T d = sc[c];
                if(!(d > T(0)))
                {
                    cfail = c; // uniform: every thread read the same d
                    break;
                }
                const T s = sqrt(d);
                const T rcp = T(1) / s;
#pragma unroll
                for(int q = 0; q < R; ++q)
                {
                    const int r = tid + q * NT;
                    if(r == c)
                        pv[q][c] = s;
                    else if(r > c && r < mp)
                    {
                        const T l = pv[q][c] * rcp;
                        pv[q][c] = l;
#pragma unroll
                        for(int cc = 0; cc < JB; ++cc)
                            if(cc > c && cc < jb && cc <= r)
                                pv[q][cc] = fma(-l, sc[cc] * rcp, pv[q][cc]);
                    }
                }
            }
        }
        // write back the factored columns (all of them on success; up to the failing
        // one otherwise, whose non-positive value is stored as LAPACK does)
        const int cdone = cfail == JB ? jb : cfail;
#pragma unroll
        for(int q = 0; q < R; ++q)
        {
            const int r = tid + q * NT;
            if(r < mp)
            {
#pragma unroll
                for(int c = 0; c < JB; ++c)
                    if(c < jb && c <= r && (c < cdone || (c == cdone && r == cdone)))
                        at(j0 + r, j0 + c) = pv[q][c];
                if(r >= jb && cfail == JB)
                {
#pragma unroll
                    for(int c = 0; c < JB; ++c)
                        sL[(size_t)(r - jb) * LDL + c] = pv[q][c];
                }
            }
        }
        if(cfail != JB)
        {
            inf = j0 + cfail + 1;
            break;
        }
        __syncthreads();
        // trailing update A22 -= L21 L21' (lower triangle only)
        const int nt = mp - jb;
        for(int t0 = 0; t0 < nt; t0 += TN)
        {
            T acc[R][TN];
#pragma unroll
            for(int q = 0; q < R; ++q)
            {
                const int rt = tid + q * NT - jb;
#pragma unroll
                for(int t = 0; t < TN; ++t)
                    acc[q][t] = (rt >= 0 && rt < nt && t0 + t <= rt)
                                    ? at(j0 + jb + rt, j0 + jb + t0 + t)
                                    : T(0);
            }
#pragma unroll
            for(int k = 0; k < JB; ++k)
            {
                if(k < jb)
                {
                    T lk[TN];
#pragma unroll
                    for(int t = 0; t < TN; ++t)
                        lk[t] = t0 + t < nt ? sL[(size_t)(t0 + t) * LDL + k] : T(0);
#pragma unroll
                    for(int q = 0; q < R; ++q)
#pragma unroll
                        for(int t = 0; t < TN; ++t)
                            acc[q][t] = fma(-pv[q][k], lk[t], acc[q][t]);
                }
            }
#pragma unroll
            for(int q = 0; q < R; ++q)
            {
                const int rt = tid + q * NT - jb;
                if(rt >= 0 && rt < nt)
                {
#pragma unroll
                    for(int t = 0; t < TN; ++t)
                        if(t0 + t <= rt)
                            at(j0 + jb + rt, j0 + jb + t0 + t) = acc[q][t];
                }
            }
        }
        __syncthreads();
    }
    if(tid == 0)
        info[b] = inf;
}

// ---------------------------------------------------------------------------------------
// Small orders (n <= N, N = 32 or 64): one thread per row, the row's lower-triangle
// entries in registers for the whole factorisation, one CTA barrier per column.
// Rolled column loop: at step c, v[i] holds A(r, c + i) of this thread's row r, so the
// active column is always v[0] and the rank-1 update writes column c+1+i into v[i].  At
// step c every row r >= c publishes A(r, c) (already updated by steps < c) at slot r-c of
// a double-buffered column vector, the diagonal row also publishes sqrt and 1/sqrt of its
// pivot (computed before the barrier), and after ONE barrier each row r > c forms
// l = A(r, c) / L(c, c), stores it, and updates
//   A(r, c+1+i) -= (l / L(c, c)) * A(c+1+i, c),   i = 0 .. N-2,
// reading the published column as aligned vectors.  Entries right of the diagonal are
// updated too (never stored) up to the warp's last row; beyond it they are skipped in
// groups of 8.  Each row stores its column-c entry as it is finalised.
// A non-positive or NaN pivot at step c: columns < c are final, A(c, c) keeps the updated
// value, the rest of the matrix is untouched and info = c + 1 (LAPACK dpotf2).
template <typename T, int N>
__global__ void __launch_bounds__(N, N <= 32 ? 16 : 6)
    potrf_reg_kernel(int upper, int n, Batch<T> A, int lda, int* info)
{
    // published column (slot r - c); rows of N + 4 elements keep both buffers 16-byte
    // aligned for the vector reads in FP32 and FP64
    __shared__ __align__(16) T scol[2][N + 4];
    __shared__ T sdiag[2][2];                  // sqrt(pivot), 1/sqrt(pivot)
    const int r = threadIdx.x;
    const int64_t b = blockIdx.x;
    T* a = A.at(b);
    const int64_t rs = upper ? lda : 1, cs = upper ? 1 : lda;
    auto at = [&](int i, int j) -> T& { return a[(int64_t)i * rs + (int64_t)j * cs]; };
    T v[N];
#pragma unroll
    for(int i = 0; i < N; ++i)
        v[i] = (r < n && i <= r) ? at(r, i) : T(0);
    int inf = 0;
#pragma unroll 1
    for(int c = 0; c < n; ++c)
    {
        const int buf = c & 1;
        if(r == c)
        {
            const T d = v[0];
            const bool ok = d > T(0);
            const T sq = ok ? sqrt(d) : d;
            sdiag[buf][0] = sq;
            sdiag[buf][1] = ok ? T(1) / sq : T(0);
            at(c, c) = sq; // LAPACK also stores a failing pivot as it was computed
        }
        else if(r > c && r < n)
            scol[buf][r - c - 1] = v[0];
        __syncthreads();
        const T sq = sdiag[buf][0];
        if(!(sq > T(0)))
        {
            inf = c + 1;
            break;
        }
        const T rcp = sdiag[buf][1];
        if(r > c && r < n)
        {
            const T l = v[0] * rcp;
            at(r, c) = l;
            const T lr = l * rcp;
            const T* col = scol[buf];
            // only columns up to the warp's last row matter: groups of 8 registers above
            // that are skipped (the branch is uniform across the warp)
            const int lim = min(32 * (r >> 5) + 31, n - 1) - c - 1;
#pragma unroll
            for(int g = 0; g < N; g += 8)
            {
                if(g > lim)
                    break;
                if constexpr(sizeof(T) == 8)
                {
#pragma unroll
                    for(int i = g; i < g + 8; i += 2)
                    {
                        const double2 t = *reinterpret_cast<const double2*>(col + i);
                        if(i + 1 < N)
                            v[i] = fma(-lr, t.x, v[i + 1]);
                        if(i + 2 < N)
                            v[i + 1] = fma(-lr, t.y, v[i + 2]);
                    }
                }
                else
                {
#pragma unroll
                    for(int i = g; i < g + 8; i += 4)
                    {
                        const float4 t = *reinterpret_cast<const float4*>(col + i);
                        const float e[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
                        for(int u = 0; u < 4; ++u)
                            if(i + u + 1 < N)
                                v[i + u] = fmaf(-lr, e[u], v[i + u + 1]);
                    }
                }
            }
        }
    }
    if(r == 0)
        info[b] = inf;
}

} // namespace rsb
