// mixed.cu -- mixed-precision batched solver with iterative refinement (dsgesv).
//
// No counterpart in the reference (rocSOLVER has no mixed-precision gesv).  Semantics are
// LAPACK dsgesv's (the CPU analogue the reference's host oracle library provides):
//   ITER >= 0 : refinement converged after ITER corrections, A unchanged, X solution;
//   ITER = -2 : A, B or a residual overflows in FP32;  ITER = -3 : the FP32 LU is singular;
//   ITER = -(ITERMAX+1): no convergence within ITERMAX corrections;
//   ITER = -1 : refinement not attempted (shape outside the fused refinement kernel);
//   for ITER < 0 the system is re-solved in FP64 (A overwritten by its LU, ipiv/info from
//   the FP64 factorisation, X = A^{-1} B).  B is never modified.
// Stopping rule (LAPACK dsgesv): every column satisfies ||r||_inf <= ||x||_inf * cte with
// cte = ||A||_inf * eps * sqrt(n), eps = 2^-53.
//
// Pipeline (all on the handle's stream, no host synchronisation):
//   1. convert : A -> FP32 copy in the workspace, overflow flags, info = iter = 0
//   2. sgetrf  : FP32 LU of the copy (the CTA LU kernels of getrf in FP32, with the trailing
//                updates as split-TF32 tensor products: FP32-level accuracy)
//   3. refine  : one CTA per matrix: x = LU32^{-1} b, then r = b - A x in FP64 (A read in
//                FP64), d = LU32^{-1} r in FP32, x += d, until the stopping rule holds
//   4. fallback: FP64 getrf + getrs gated to the members whose refinement failed.
#include <math.h>

#include "handle.h"
#include "launch.h"
#include "logger.h"
#include "trsv.cuh"

namespace rsb {

// LAPACK dsgesv allows ITERMAX = 30 corrections; this solver stops at 10 (ITER = -11 then),
// the iteration budget of the benchmarked configuration: every pass re-reads A in FP64 and
// the FP32 factors (~0.8 MB per member at n = 256), and a member still short of the
// stopping rule after 10 passes is re-solved in FP64 for about the cost of 5 more passes.
// ITER values therefore differ from LAPACK's for members that would converge in 11-30
// corrections (they take the FP64 path here).
constexpr int DSGESV_ITERMAX = 10;
// refinement solves use inverted diagonal blocks up to this order (their shared memory
// grows as n); larger orders use the staged-block substitution
constexpr int REFINE_BLOCKINV_MAXN = 512;
// CTAs of the refinement kernel resident per SM: their A (FP64) and FP32 factors should
// stay in L2 between iterations
#ifndef REFINE_CTAS_PER_SM
#define REFINE_CTAS_PER_SM 2
#endif
// threads per refinement CTA (rows of at most half this order use two threads per row in
// the residual)
#ifndef REFINE_NT
#define REFINE_NT 256
#endif
// 8-column load batches in flight per residual row: 2 measured fastest on B200 at n = 256
// (dsgesv step 4.10 ms; 1 batch 4.50 ms, 4 batches 4.39 ms with register spills)
#ifndef REFINE_RES_UNROLL
#define REFINE_RES_UNROLL 2
#endif
constexpr int kResUnroll = REFINE_RES_UNROLL;

// A -> FP32 copy (ld n), FP32 overflow flag (LAPACK dsgesv: any |a_ij| > FLT_MAX sends
// the member to the FP64 path), info = iter = 0.  One CTA per matrix, threads over rows,
// 8 columns of loads in flight per thread.
__global__ void __launch_bounds__(256)
    dsgesv_convert_kernel(int n, Batch<double> A, int lda, float* a32, int* flag, int* info,
                          int* iter)
{
    __shared__ int ovf;
    const int64_t b = blockIdx.x;
    const double* a = A.at(b);
    float* s = a32 + (size_t)b * n * n;
    if(threadIdx.x == 0)
        ovf = 0;
    __syncthreads();
    int ov = 0;
    for(int i = threadIdx.x; i < n; i += blockDim.x)
    {
        int j = 0;
        for(; j + 8 <= n; j += 8)
        {
            double v[8];
#pragma unroll
            for(int u = 0; u < 8; ++u)
                v[u] = a[ix(i, j + u, lda)];
#pragma unroll
            for(int u = 0; u < 8; ++u)
            {
                ov |= fabs(v[u]) > (double)FLT_MAX;
                s[ix(i, j + u, n)] = (float)v[u];
            }
        }
        for(; j < n; ++j)
        {
            const double v = a[ix(i, j, lda)];
            ov |= fabs(v) > (double)FLT_MAX;
            s[ix(i, j, n)] = (float)v;
        }
    }
    if(ov)
        atomicOr(&ovf, 1);
    __syncthreads();
    if(threadIdx.x == 0)
    {
        flag[b] = ovf;
        info[b] = 0;
        iter[b] = 0;
    }
}

// block-wide max of a non-negative value; all threads get the result
template <int NT>
__device__ __forceinline__ double block_max(double v, double* red)
{
    for(int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = red[0];
#pragma unroll
    for(int w = 1; w < NT / 32; ++w)
        m = fmax(m, red[w]);
    return m;
}

// ---- triangular solves with the FP32 factors through inverted 32x32 diagonal blocks
constexpr int BI_LD = 33;
constexpr int BI_ELEMS = 32 * BI_LD;

// Invert the diagonal blocks of the FP32 LU once per matrix: blocks 0..nblk-1 of L (unit
// lower) and nblk..2*nblk-1 of U (upper).  One warp per block: the block is staged
// row-major in its slot, lane j computes column j of the inverse by substitution in
// registers, then the lanes overwrite the block with the inverse.  Partial blocks are
// padded with the identity.
template <int NT>
__device__ void invert_diag_blocks(const float* lu, int n, float* sinv)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nblk = (n + 31) / 32;
    for(int t = warp; t < 2 * nblk; t += NT / 32)
    {
        const bool upper = t >= nblk;
        const int kb = (upper ? t - nblk : t) * 32, nb = min(32, n - kb);
        float* blk = sinv + t * BI_ELEMS;
        {
            // all 32 loads of the block column strip in flight before the stores
            const int i = lane;
            float v[32];
#pragma unroll
            for(int k = 0; k < 32; ++k)
            {
                if(i >= nb || k >= nb)
                    v[k] = i == k ? 1.f : 0.f;
                else if(!upper)
                    v[k] = i > k ? lu[(kb + i) + (size_t)(kb + k) * n] : (i == k ? 1.f : 0.f);
                else
                    v[k] = i <= k ? lu[(kb + i) + (size_t)(kb + k) * n] : 0.f;
            }
#pragma unroll
            for(int k = 0; k < 32; ++k)
                blk[i * BI_LD + k] = v[k];
        }
        __syncwarp();
        float x[32];
#pragma unroll
        for(int i = 0; i < 32; ++i)
            x[i] = i == lane ? 1.f : 0.f;
        if(!upper)
        {
#pragma unroll
            for(int k = 0; k < 32; ++k)
#pragma unroll
                for(int i = k + 1; i < 32; ++i)
                    x[i] = fmaf(-blk[i * BI_LD + k], x[k], x[i]);
        }
        else
        {
#pragma unroll
            for(int k = 31; k >= 0; --k)
            {
                x[k] = x[k] / blk[k * BI_LD + k];
#pragma unroll
                for(int i = 0; i < k; ++i)
                    x[i] = fmaf(-blk[i * BI_LD + k], x[k], x[i]);
            }
        }
        __syncwarp();
#pragma unroll
        for(int i = 0; i < 32; ++i)
            blk[i * BI_LD + lane] = x[i];
        __syncwarp();
    }
}

// Solve (forward: L, unit lower; else U) for nc columns of s (ld n) using the inverted
// diagonal blocks: per 32-block, warp 0 applies the block inverse (a 32x32 mat-vec, no
// serial chain), then all threads apply the block to the remaining rows.
template <int NT, int NRC>
__device__ void blockinv_sweep(bool forward, const float* lu, int n, const float* sinv,
                               float* s, int nc)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nblk = (n + 31) / 32;
    for(int bi = 0; bi < nblk; ++bi)
    {
        const int blkid = forward ? bi : nblk - 1 - bi;
        const int kb = blkid * 32, nb = min(32, n - kb);
        const float* inv = sinv + (forward ? blkid : nblk + blkid) * BI_ELEMS;
        if(warp == 0)
        {
            float y[NRC];
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                y[c] = 0.f;
#pragma unroll 8
            for(int j = 0; j < 32; ++j)
            {
                const float mij = inv[lane * BI_LD + j];
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                    if(c < nc && j < nb)
                        y[c] = fmaf(mij, s[kb + j + c * n], y[c]);
            }
            __syncwarp();
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                if(c < nc && lane < nb)
                    s[kb + lane + c * n] = y[c];
        }
        __syncthreads();
        const int r0 = forward ? kb + nb : 0;
        const int r1 = forward ? n : kb;
        for(int i = r0 + tid; i < r1; i += NT)
        {
            float acc[NRC];
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                acc[c] = c < nc ? s[i + c * n] : 0.f;
            if(nb == 32)
            {
                float mv[32];
#pragma unroll
                for(int k = 0; k < 32; ++k)
                    mv[k] = lu[i + (size_t)(kb + k) * n];
#pragma unroll
                for(int k = 0; k < 32; ++k)
#pragma unroll
                    for(int c = 0; c < NRC; ++c)
                        acc[c] = fmaf(-mv[k], s[kb + k + c * n], acc[c]);
            }
            else
            {
                for(int k = 0; k < nb; ++k)
                {
                    const float mik = lu[i + (size_t)(kb + k) * n];
#pragma unroll
                    for(int c = 0; c < NRC; ++c)
                        acc[c] = fmaf(-mik, s[kb + k + c * n], acc[c]);
                }
            }
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                if(c < nc)
                    s[i + c * n] = acc[c];
        }
        __syncthreads();
    }
}

// blockinv_sweep for n <= NT with a fixed row per thread (row = threadIdx.x), so that the
// factor strip a thread needs for block bi+1 can be loaded as soon as block bi's update has
// consumed the previous one: the loads overlap the barrier and the next diagonal-block
// product instead of following them.
template <int NT, int NRC>
__device__ void blockinv_sweep_pf(bool forward, const float* lu, int n, const float* sinv,
                                  float* s, int nc)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nblk = (n + 31) / 32;
    const int i = tid;
    // this thread's row of the factor strip of sweep step bi (columns of block bi)
    auto load_strip = [&](int bi, float (&v)[32]) {
        const int blkid = forward ? bi : nblk - 1 - bi;
        const int kb = blkid * 32, nb = min(32, n - kb);
        const bool act = forward ? (i >= kb + nb && i < n) : (i < kb);
        if(act)
        {
#pragma unroll
            for(int k = 0; k < 32; ++k)
                v[k] = k < nb ? lu[i + (size_t)(kb + k) * n] : 0.f;
        }
    };
    float mv[32];
    load_strip(0, mv);
    for(int bi = 0; bi < nblk; ++bi)
    {
        const int blkid = forward ? bi : nblk - 1 - bi;
        const int kb = blkid * 32, nb = min(32, n - kb);
        const float* inv = sinv + (forward ? blkid : nblk + blkid) * BI_ELEMS;
        if(warp == 0)
        {
            float y0[NRC], y1[NRC];
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                y0[c] = y1[c] = 0.f;
#pragma unroll 4
            for(int j = 0; j < 32; j += 2)
            {
                const float m0 = inv[lane * BI_LD + j], m1 = inv[lane * BI_LD + j + 1];
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                    if(c < nc)
                    {
                        if(j < nb)
                            y0[c] = fmaf(m0, s[kb + j + c * n], y0[c]);
                        if(j + 1 < nb)
                            y1[c] = fmaf(m1, s[kb + j + 1 + c * n], y1[c]);
                    }
            }
            __syncwarp();
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                if(c < nc && lane < nb)
                    s[kb + lane + c * n] = y0[c] + y1[c];
        }
        __syncthreads();
        const bool act = forward ? (i >= kb + nb && i < n) : (i < kb);
        if(act)
        {
            float acc[NRC];
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                acc[c] = c < nc ? s[i + c * n] : 0.f;
#pragma unroll
            for(int k = 0; k < 32; ++k)
                if(k < nb)
#pragma unroll
                    for(int c = 0; c < NRC; ++c)
                        acc[c] = fmaf(-mv[k], s[kb + k + c * n], acc[c]);
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                if(c < nc)
                    s[i + c * n] = acc[c];
        }
        // the next step's strip (its rows are a subset of this step's, or the same); a
        // second strip in flight does not fit the register budget of two CTAs per SM
        if(bi + 1 < nblk)
            load_strip(bi + 1, mv);
        __syncthreads();
    }
}

// r = b - A x for right-hand sides c0..c0+nc-1 in FP64, threads over rows (column-major A:
// a warp reads 32 consecutive rows of a column), 8 columns of loads in flight per thread.
// With rowsum, also returns this thread's largest row sum of |A| (for ||A||_inf).
template <int NT, int NRC>
__device__ double residual_rows(const double* a, int lda, const double* bb, int ldb,
                                const double* xs, double* rs, int n, int c0, int nc,
                                bool rowsum)
{
    double amax = 0.0;
    for(int i = threadIdx.x; i < n; i += NT)
    {
        double acc[NRC];
#pragma unroll
        for(int c = 0; c < NRC; ++c)
            acc[c] = c < nc ? bb[ix(i, c0 + c, ldb)] : 0.0;
        double asum = 0.0;
        int j = 0;
#pragma unroll kResUnroll
        for(; j + 8 <= n; j += 8)
        {
            double v[8];
#pragma unroll
            for(int u = 0; u < 8; ++u)
                v[u] = a[ix(i, j + u, lda)];
#pragma unroll
            for(int u = 0; u < 8; ++u)
            {
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                    if(c < nc)
                        acc[c] = fma(-v[u], xs[j + u + (size_t)(c0 + c) * n], acc[c]);
                if(rowsum)
                    asum += fabs(v[u]);
            }
        }
        for(; j < n; ++j)
        {
            const double v = a[ix(i, j, lda)];
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                if(c < nc)
                    acc[c] = fma(-v, xs[j + (size_t)(c0 + c) * n], acc[c]);
            if(rowsum)
                asum += fabs(v);
        }
#pragma unroll
        for(int c = 0; c < NRC; ++c)
            if(c < nc)
                rs[i + (size_t)(c0 + c) * n] = acc[c];
        amax = fmax(amax, asum);
    }
    return amax;
}

// residual_rows with two threads per row (n <= NT/2): thread t takes row t mod NT/2 and
// half t div NT/2 of the columns; the second half's partial sums meet the first's through
// shared memory (part, n*NRC doubles).  Same arithmetic per half as residual_rows; the two
// halves are added once at the end.
template <int NT, int NRC>
__device__ double residual_rows_split(const double* a, int lda, const double* bb, int ldb,
                                      const double* xs, double* rs, double* part, int n,
                                      int c0, int nc, bool rowsum)
{
    constexpr int H = NT / 2;
    const int i = threadIdx.x % H, h = threadIdx.x / H;
    const int half = (n + 1) / 2;
    const int j0 = h ? half : 0, j1 = h ? n : half;
    double acc[NRC];
    double asum = 0.0;
#pragma unroll
    for(int c = 0; c < NRC; ++c)
        acc[c] = 0.0;
    if(i < n)
    {
        int j = j0;
#pragma unroll 2
        for(; j + 8 <= j1; j += 8)
        {
            double v[8];
#pragma unroll
            for(int u = 0; u < 8; ++u)
                v[u] = a[ix(i, j + u, lda)];
#pragma unroll
            for(int u = 0; u < 8; ++u)
            {
#pragma unroll
                for(int c = 0; c < NRC; ++c)
                    if(c < nc)
                        acc[c] = fma(-v[u], xs[j + u + (size_t)(c0 + c) * n], acc[c]);
                if(rowsum)
                    asum += fabs(v[u]);
            }
        }
        for(; j < j1; ++j)
        {
            const double v = a[ix(i, j, lda)];
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                if(c < nc)
                    acc[c] = fma(-v, xs[j + (size_t)(c0 + c) * n], acc[c]);
            if(rowsum)
                asum += fabs(v);
        }
        if(h)
        {
#pragma unroll
            for(int c = 0; c < NRC; ++c)
                if(c < nc)
                    part[i + c * n] = acc[c];
            part[(size_t)NRC * n + i] = asum;
        }
    }
    __syncthreads();
    double amax = 0.0;
    if(!h && i < n)
    {
#pragma unroll
        for(int c = 0; c < NRC; ++c)
            if(c < nc)
                rs[i + (size_t)(c0 + c) * n] = bb[ix(i, c0 + c, ldb)] + (acc[c] + part[i + c * n]);
        amax = asum + part[(size_t)NRC * n + i];
    }
    __syncthreads();
    return amax;
}

template <int NT, int NRC>
__global__ void __launch_bounds__(NT, REFINE_CTAS_PER_SM)
    dsgesv_refine_kernel(int n, int nrhs, Batch<double> A, int lda, const float* lu32,
                         const int* ipiv, int64_t strideP, Batch<double> B, int ldb,
                         Batch<double> X, int ldx, int* flag, const int* info32, int* iter,
                         int itermax)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* xs = reinterpret_cast<double*>(smem_raw);   // n x nrhs
    double* rs = xs + (size_t)n * nrhs;                    // n x nrhs
    double* red = rs + (size_t)n * nrhs;                   // NT/32
    float* sdiag = reinterpret_cast<float*>(red + NT / 32); // staged diagonal blocks
    const bool blockinv = n <= REFINE_BLOCKINV_MAXN;
    float* s32 = sdiag + (blockinv ? SDIAG_ELEMS : sweep_scratch<NT>()); // n x NRC
    int* perm = reinterpret_cast<int*>(s32 + (size_t)n * NRC);
    float* sinv = reinterpret_cast<float*>(perm + ((n + 3) & ~3)); // [2*nblk][32x33]
    double* part = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(sinv + (blockinv ? 2 * ((n + 31) / 32) * BI_ELEMS : 0))
         + 15)
        & ~uintptr_t(15)); // (NRC+1) x n doubles, split residual rows
    const bool split = 2 * n <= NT;
    __shared__ int bad;

    const int64_t b = blockIdx.x;
    const int tid = threadIdx.x;
    if(flag[b] != 0 || info32[b] != 0)
    {
        __syncthreads();
        if(tid == 0)
        {
            iter[b] = flag[b] != 0 ? -2 : -3;
            flag[b] = 1;
        }
        return;
    }
    const double* a = A.at(b);
    const double* bb = B.at(b);
    double* x = X.at(b);
    const float* lu = lu32 + (size_t)b * n * n;
    if(blockinv)
        invert_diag_blocks<NT>(lu, n, sinv);
    build_perm(ipiv + b * strideP, n, perm);
    const int tot = n * nrhs;
    for(int e = tid; e < tot; e += NT)
    {
        const int i = e % n, c = e / n;
        rs[e] = bb[ix(i, c, ldb)];
        xs[e] = 0.0;
    }
    if(tid == 0)
        bad = 0;
    __syncthreads();
    double cte = 0.0;
    for(int it = 0;; ++it)
    {
        // ---- correction d = (LU32)^{-1} P r in FP32, x += d
        for(int c0 = 0; c0 < nrhs; c0 += NRC)
        {
            const int nc = min(NRC, nrhs - c0);
            for(int e = tid; e < n * nc; e += NT)
            {
                const int i = e % n, c = e / n;
                const double v = rs[perm[i] + (c0 + c) * n];
                if(v > (double)FLT_MAX || v < -(double)FLT_MAX)
                    bad = 1;
                s32[i + c * n] = (float)v;
            }
            __syncthreads();
            if(blockinv && n <= NT)
            {
                blockinv_sweep_pf<NT, NRC>(true, lu, n, sinv, s32, nc);
                blockinv_sweep_pf<NT, NRC>(false, lu, n, sinv, s32, nc);
            }
            else if(blockinv)
            {
                blockinv_sweep<NT, NRC>(true, lu, n, sinv, s32, nc);
                blockinv_sweep<NT, NRC>(false, lu, n, sinv, s32, nc);
            }
            else
            {
                block_sweep<float, NT, NRC, true>(true, TriView<float>{lu, 1, n}, n, s32, nc,
                                            sdiag);
                block_sweep<float, NT, NRC, false>(false, TriView<float>{lu, 1, n}, n, s32, nc,
                                            sdiag);
            }
            for(int e = tid; e < n * nc; e += NT)
            {
                const int i = e % n, c = e / n;
                xs[i + (c0 + c) * n] += (double)s32[i + c * n];
            }
            __syncthreads();
        }
        if(bad)
        {
            if(tid == 0)
            {
                iter[b] = -2;
                flag[b] = 1;
            }
            return;
        }
        // ---- residual r = b - A x in FP64; the first pass also yields ||A||_inf
        double amax = 0.0;
        for(int c0 = 0; c0 < nrhs; c0 += NRC)
            amax = fmax(amax,
                        split ? residual_rows_split<NT, NRC>(a, lda, bb, ldb, xs, rs, part, n, c0,
                                                             min(NRC, nrhs - c0),
                                                             it == 0 && c0 == 0)
                              : residual_rows<NT, NRC>(a, lda, bb, ldb, xs, rs, n, c0,
                                                       min(NRC, nrhs - c0), it == 0 && c0 == 0));
        if(it == 0)
            cte = block_max<NT>(amax, red) * (DBL_EPSILON * 0.5) * sqrt((double)n);
        __syncthreads();
        // ---- stopping rule (LAPACK dsgesv): every column, ||r||_inf <= ||x||_inf * cte
        bool conv = true;
        for(int c = 0; c < nrhs; ++c)
        {
            double xm = 0.0, rm = 0.0;
            for(int i = tid; i < n; i += NT)
            {
                xm = fmax(xm, fabs(xs[i + c * n]));
                rm = fmax(rm, fabs(rs[i + c * n]));
            }
            const double XN = block_max<NT>(xm, red);
            const double RN = block_max<NT>(rm, red);
            if(RN > XN * cte)
                conv = false;
        }
        if(conv)
        {
            for(int e = tid; e < tot; e += NT)
            {
                const int i = e % n, c = e / n;
                x[ix(i, c, ldx)] = xs[e];
            }
            if(tid == 0)
                iter[b] = it;
            return;
        }
        if(it == itermax)
        {
            if(tid == 0)
            {
                iter[b] = -(itermax + 1);
                flag[b] = 1;
            }
            return;
        }
    }
}

// X = B for the gated members (the FP64 fallback restarts from B)
__global__ void copy_gated_kernel(int n, int nrhs, Batch<double> B, int ldb, Batch<double> X,
                                  int ldx, Gate gate)
{
    const int64_t b = blockIdx.x;
    if(gate.skip(b))
        return;
    const double* s = B.at(b);
    double* d = X.at(b);
    for(int e = threadIdx.x; e < n * nrhs; e += blockDim.x)
    {
        const int i = e % n, c = e / n;
        d[ix(i, c, ldx)] = s[ix(i, c, ldb)];
    }
}

// mark every member for the FP64 path with ITER = -1 (refinement not attempted)
__global__ void mark_all_kernel(int bc, int* flag, int* info, int* iter)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < bc)
    {
        flag[i] = 1;
        info[i] = 0;
        iter[i] = -1;
    }
}

static size_t refine_smem(int n, int nrhs, int NRC, int NT)
{
    const size_t nblk = (n + 31) / 32;
    const size_t inv = n <= REFINE_BLOCKINV_MAXN ? 2 * nblk * BI_ELEMS : 0;
    const size_t part = 2 * n <= NT ? (size_t)(NRC + 1) * n : 0;
    return sizeof(double) * (2 * (size_t)n * nrhs + NT / 32)
           + sizeof(float) * ((size_t)n * NRC + (inv ? SDIAG_ELEMS : (size_t)sweep_scratch<REFINE_NT>())
                              + inv)
           + sizeof(int) * (size_t)((n + 3) & ~3) + sizeof(double) * part + 16;
}

size_t dsgesv_workspace(int n, int nrhs, int bc)
{
    (void)nrhs;
    return ws_round(sizeof(float) * (size_t)n * n * bc) + 3 * ws_round(sizeof(int) * bc);
}

rocblas_status launch_dsgesv(cudaStream_t s, int n, int nrhs, Batch<double> A, int lda,
                             int* ipiv, int64_t strideP, Batch<double> B, int ldb,
                             Batch<double> X, int ldx, int* iter, int* info, int bc, void* ws)
{
    char* p = static_cast<char*>(ws);
    float* a32 = reinterpret_cast<float*>(p);
    p += ws_round(sizeof(float) * (size_t)n * n * bc);
    int* flag = reinterpret_cast<int*>(p);
    p += ws_round(sizeof(int) * bc);
    int* info32 = reinterpret_cast<int*>(p);

    constexpr int NT = REFINE_NT;
    const int NRC = nrhs == 1 ? 1 : 4;
    const size_t smem = refine_smem(n, nrhs, NRC, NT);
    const bool refine_ok = smem <= 200 * 1024 && n <= MAX_CTA_ROWS;
    if(refine_ok)
    {
        {
            RSB_LOG_KERNEL("dsgesv_convert_kernel");
            dsgesv_convert_kernel<<<bc, 256, 0, s>>>(n, A, lda, a32, flag, info, iter);
        }
        if(cudaGetLastError() != cudaSuccess)
            return rocblas_status_internal_error;
        rocblas_status st = launch_getrf<float>(s, n, n, strided<float>(a32, (int64_t)n * n), n,
                                                ipiv, strideP, info32, bc, true, Gate{flag, 0},
                                                true);
        if(st != rocblas_status_success)
            return st;
        RSB_LOG_KERNEL("dsgesv_refine_kernel");
        if(NRC == 1)
        {
            auto k = dsgesv_refine_kernel<NT, 1>;
            if(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem)
               != cudaSuccess)
                return rocblas_status_internal_error;
            k<<<bc, NT, smem, s>>>(n, nrhs, A, lda, a32, ipiv, strideP, B, ldb, X, ldx, flag,
                                   info32, iter, DSGESV_ITERMAX);
        }
        else
        {
            auto k = dsgesv_refine_kernel<NT, 4>;
            if(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem)
               != cudaSuccess)
                return rocblas_status_internal_error;
            k<<<bc, NT, smem, s>>>(n, nrhs, A, lda, a32, ipiv, strideP, B, ldb, X, ldx, flag,
                                   info32, iter, DSGESV_ITERMAX);
        }
        if(cudaGetLastError() != cudaSuccess)
            return rocblas_status_internal_error;
    }
    else
    {
        mark_all_kernel<<<(bc + 255) / 256, 256, 0, s>>>(bc, flag, info, iter);
    }
    // FP64 fallback for the flagged members
    const Gate g{flag, 1};
    rocblas_status st = launch_getrf<double>(s, n, n, A, lda, ipiv, strideP, info, bc, true, g);
    if(st != rocblas_status_success)
        return st;
    copy_gated_kernel<<<bc, 256, 0, s>>>(n, nrhs, B, ldb, X, ldx, g);
    if(cudaGetLastError() != cudaSuccess)
        return rocblas_status_internal_error;
    return launch_getrs<double>(s, 0, n, nrhs, A, lda, ipiv, strideP, X, ldx, info, bc, g);
}

} // namespace rsb
