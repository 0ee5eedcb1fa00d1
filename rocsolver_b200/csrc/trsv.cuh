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

// Scratch (elements) block_sweep needs: one inverted 32x32 diagonal block per warp, and
// the solved block's values for up to 32 right-hand sides.
template <int NT>
__host__ __device__ constexpr int sweep_scratch()
{
    return (NT / 32) * SDIAG_ELEMS + 32 * 32;
}

// Invert the diagonal block M(kb.., kb..) (order nb <= 32, padded with the identity) with
// one warp, in place in blk (row-major, blk[i*SDIAG_LD + k]): the block is staged
// coalesced along M's contiguous direction, then lane j computes column j of the inverse
// eight rows at a time (LOWER: top-down, else bottom-up): the rows already finished
// contribute through shared memory, the eight new rows are solved in registers, written
// over the block's rows once every lane has read them, and the next eight follow.  Few
// registers, so the sweep kernels keep their occupancy.  unit: unit diagonal.
template <typename T, bool LOWER>
__device__ __forceinline__ void invert_block(bool unit, TriView<T> M, int kb, int nb, T* blk)
{
    const int lane = threadIdx.x & 31;
    // 8 loads per lane issued before their stores (overlapped latency)
    for(int e0 = lane; e0 < 32 * 32; e0 += 8 * 32)
    {
        T v[8];
#pragma unroll
        for(int u = 0; u < 8; ++u)
        {
            const int e = e0 + 32 * u;
            const int i = M.rs == 1 ? (e & 31) : (e >> 5); // M's contiguous direction first
            const int k = M.rs == 1 ? (e >> 5) : (e & 31);
            if(i >= nb || k >= nb)
                v[u] = i == k ? T(1) : T(0);
            else if(i == k)
                v[u] = unit ? T(1) : M(kb + i, kb + k);
            else
                v[u] = (LOWER ? i > k : i < k) ? M(kb + i, kb + k) : T(0);
        }
#pragma unroll
        for(int u = 0; u < 8; ++u)
        {
            const int e = e0 + 32 * u;
            const int i = M.rs == 1 ? (e & 31) : (e >> 5);
            const int k = M.rs == 1 ? (e >> 5) : (e & 31);
            blk[i * SDIAG_LD + k] = v[u];
        }
    }
    __syncwarp();
#pragma unroll 1
    for(int rb = 0; rb < 4; ++rb)
    {
        const int r0 = LOWER ? 8 * rb : 24 - 8 * rb; // first row of this group
        T x[8];
#pragma unroll
        for(int u = 0; u < 8; ++u)
            x[u] = r0 + u == lane ? T(1) : T(0);
        // finished rows: above the group (LOWER) or below it
        const int k0 = LOWER ? 0 : r0 + 8, k1 = LOWER ? r0 : 32;
#pragma unroll 4
        for(int k = k0; k < k1; ++k)
        {
            const T xk = blk[k * SDIAG_LD + lane];
#pragma unroll
            for(int u = 0; u < 8; ++u)
                x[u] = fma(-blk[(r0 + u) * SDIAG_LD + k], xk, x[u]);
        }
        // the group's own rows
        if constexpr(LOWER)
        {
#pragma unroll
            for(int u = 0; u < 8; ++u)
            {
#pragma unroll
                for(int v = 0; v < u; ++v)
                    x[u] = fma(-blk[(r0 + u) * SDIAG_LD + r0 + v], x[v], x[u]);
                if(!unit)
                    x[u] = x[u] / blk[(r0 + u) * SDIAG_LD + r0 + u];
            }
        }
        else
        {
#pragma unroll
            for(int u = 7; u >= 0; --u)
            {
#pragma unroll
                for(int v = u + 1; v < 8; ++v)
                    x[u] = fma(-blk[(r0 + u) * SDIAG_LD + r0 + v], x[v], x[u]);
                if(!unit)
                    x[u] = x[u] / blk[(r0 + u) * SDIAG_LD + r0 + u];
            }
        }
        __syncwarp();
#pragma unroll
        for(int u = 0; u < 8; ++u)
            blk[(r0 + u) * SDIAG_LD + lane] = x[u];
        __syncwarp();
    }
}

// Solve M x = b in place for the nc columns of sb (ld = n).  FORWARD: M lower
// (substitution top-down), else M upper (bottom-up).  unit: unit diagonal.
// sinv: shared scratch of sweep_scratch<NT>() elements.  Must be called by all NT threads.
// The 32-wide diagonal blocks are taken in chunks of NT/32: every warp inverts one block
// of the chunk in parallel (off the sweep's serial path), then per block the threads
// apply the inverse (a 32x32 product, no serial chain) and all threads apply the block's
// columns to the remaining rows with independent (unrolled) factor loads.  The block
// product is spread over all threads (one row and right-hand side each).  Explicit
// inverses of the diagonal blocks are also what the reference's batched trsm uses
// (rocBLAS trsm with invA).
template <typename T, int NT, int NRC, bool FORWARD>
__device__ void block_sweep(bool unit, TriView<T> M, int n, T* sb, int nc, T* sinv)
{
    constexpr bool forward = FORWARD;
    constexpr int NW = NT / 32;
    static_assert(NRC <= 32, "right-hand sides per pass");
    const int tid = threadIdx.x, warp = tid >> 5;
    const int nblk = (n + 31) / 32;
    T* sy = sinv + NW * SDIAG_ELEMS; // [NRC][32]
    for(int cb = 0; cb < nblk; cb += NW)
    {
        {
            const int bi = cb + warp;
            if(bi < nblk)
            {
                const int kb = forward ? bi * 32 : (nblk - 1 - bi) * 32;
                invert_block<T, FORWARD>(unit, M, kb, min(32, n - kb), sinv + warp * SDIAG_ELEMS);
            }
        }
        __syncthreads();
        const int cend = min(cb + NW, nblk);
        for(int bi = cb; bi < cend; ++bi)
        {
            const int kb = forward ? bi * 32 : (nblk - 1 - bi) * 32;
            const int nb = min(32, n - kb);
            const T* inv = sinv + (bi - cb) * SDIAG_ELEMS;
            // y = inv * b_block for every right-hand side: one output (row, rhs) per thread,
            // written to the side buffer sy so that no thread overwrites an input
            for(int o = tid; o < 32 * nc; o += NT)
            {
                const int row = o & 31, c = o >> 5;
                T y0 = T(0), y1 = T(0);
#pragma unroll 4
                for(int j = 0; j < 32; j += 2)
                {
                    if(j < nb)
                        y0 = fma(inv[row * SDIAG_LD + j], sb[kb + j + c * n], y0);
                    if(j + 1 < nb)
                        y1 = fma(inv[row * SDIAG_LD + j + 1], sb[kb + j + 1 + c * n], y1);
                }
                sy[row + 32 * c] = y0 + y1;
            }
            __syncthreads();
            for(int o = tid; o < 32 * nc; o += NT)
                if((o & 31) < nb)
                    sb[kb + (o & 31) + (o >> 5) * n] = sy[o];
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
                            acc[c] = fma(-mv[k], sy[k + 32 * c], acc[c]);
                }
                else
                {
                    for(int k = 0; k < nb; ++k)
                    {
                        const T mik = M(i, kb + k);
#pragma unroll
                        for(int c = 0; c < NRC; ++c)
                            acc[c] = fma(-mik, sy[k + 32 * c], acc[c]);
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
        {
            RSB_CHECK_PIV(piv[k], n, __LINE__);
            perm[k] = piv[k] - 1;
        }
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
        staged_copy<NT, 4>(
            n * nc,
            [&](int e) {
                const int i = e % n, c = e / n;
                return x[ix((!trans && piv) ? perm[i] : i, c0 + c, ldb)];
            },
            [&](int e, T v) { sb[e] = v; });
        __syncthreads();
        if(!trans)
        {
            block_sweep<T, NT, NRC, true>(true, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
            block_sweep<T, NT, NRC, false>(false, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
        }
        else
        {
            block_sweep<T, NT, NRC, true>(false, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
            block_sweep<T, NT, NRC, false>(true, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
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
    T* sb = sdiag + sweep_scratch<NT>();
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
    staged_copy<NT, 4>(
        n * nc,
        [&](int e) {
            const int i = e % n, c = e / n;
            return RSB_AT(x, (!trans && pv) ? perm[i] : i, c0 + c, ldb, n, nrhs);
        },
        [&](int e, T v) { sb[e] = v; });
    __syncthreads();
    if(!trans)
    {
        block_sweep<T, NT, NRC, true>(true, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
        block_sweep<T, NT, NRC, false>(false, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
    }
    else
    {
        block_sweep<T, NT, NRC, true>(false, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
        block_sweep<T, NT, NRC, false>(true, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
    }
    for(int e = threadIdx.x; e < n * nc; e += NT)
    {
        const int i = e % n, c = e / n;
        const int dst = (trans && pv) ? perm[i] : i;
        RSB_AT(x, dst, c0 + c, ldb, n, nrhs) = sb[i + c * n];
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
    T* sb = sdiag + sweep_scratch<NT>();
    const int groups = (nrhs + NRC - 1) / NRC;
    const int64_t b = blockIdx.x / groups;
    const int c0 = (blockIdx.x % groups) * NRC;
    const int nc = min(NRC, nrhs - c0);
    if(skip_info && skip_info[b] != 0)
        return;
    const T* a = A.at(b);
    T* x = B.at(b);
    staged_copy<NT, 4>(
        n * nc, [&](int e) { return x[ix(e % n, c0 + e / n, ldb)]; },
        [&](int e, T v) { sb[e] = v; });
    __syncthreads();
    if(!upper)
    {
        block_sweep<T, NT, NRC, true>(false, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
        block_sweep<T, NT, NRC, false>(false, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
    }
    else
    {
        block_sweep<T, NT, NRC, true>(false, TriView<T>{a, lda, 1}, n, sb, nc, sdiag);
        block_sweep<T, NT, NRC, false>(false, TriView<T>{a, 1, lda}, n, sb, nc, sdiag);
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
    // the lower triangle packed by columns: L(i, j), i >= j, at sL[pk(j) + i - j] (half the
    // shared memory of a square tile, so twice the members per SM)
    __shared__ T sL[N * (N + 1) / 2];
    auto pk = [](int j) { return (j * (2 * N - j + 1)) / 2; };
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
    for(int e0 = r; e0 < N * N; e0 += 8 * N)
    {
        T t[8];
#pragma unroll
        for(int u = 0; u < 8; ++u)
        {
            const int e = e0 + u * N, p = e % N, q = e / N;
            const int i = upper ? q : p, j = upper ? p : q; // L(i, j), i >= j
            t[u] = (e < N * N && i < n && j <= i) ? (upper ? a[ix(j, i, lda)] : a[ix(i, j, lda)])
                                                  : T(0);
        }
#pragma unroll
        for(int u = 0; u < 8; ++u)
        {
            const int e = e0 + u * N, p = e % N, q = e / N;
            const int i = upper ? q : p, j = upper ? p : q;
            if(e < N * N && i < n && j <= i)
                sL[pk(j) + i - j] = t[u];
        }
    }
    T v[NRC];
#pragma unroll
    for(int k = 0; k < NRC; ++k)
        v[k] = (r < n && k < nc) ? x[ix(r, c0 + k, ldb)] : T(0);
    __syncthreads();
    const T rd = r < n ? T(1) / sL[pk(r)] : T(0);
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
            const T l = sL[pk(c) + r - c];
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
            const T l = sL[pk(r) + c - r];
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
