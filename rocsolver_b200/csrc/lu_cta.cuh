// lu_cta.cuh -- CTA-per-matrix blocked LU (right-looking, partial pivoting) for
// general m x n.
//
// Replaces the reference's blocked getrf (library/src/lapack/roclapack_getrf.hpp:609-752:
// getrf_panelLU :423-525, getrf_row_permutate :172-210, rocsolver_trsm_lower and the
// rocBLAS GEMM trailing update :721-732), which issues ~100 launches per call at n=256.
//
// B200 design: ONE launch, one CTA per matrix, the whole factorisation in the CTA:
//   * panel (rows j0..m-1, JB columns) resident in registers, R rows per thread; the
//     column pivot is a warp redux.sync argmax plus one __syncthreads per column (each
//     warp publishes its candidate row, so the winner's row is broadcast by the same
//     barrier); row interchanges inside the panel are lane relabellings;
//   * the panel's interchanges are applied to the other columns as ONE gather/scatter of
//     the moved rows (at most 2*JB of them) instead of JB serial swaps;
//   * U12 = L11^{-1} A12 with one thread per column (L11 broadcast from shared memory);
//   * A22 -= L21 U12 with the L21 rows still in the registers that factored them and
//     U12 broadcast from shared memory; A22 is streamed from L2/HBM once per panel.
#pragma once

#include "common.cuh"

namespace rsb {

template <typename T, int NT, int JB>
struct CtaLuSmem
{
    static constexpr int NW = NT / 32;
    // byte offsets inside dynamic shared memory
    static __host__ __device__ size_t bytes(int cw, int R)
    {
        using K = typename KeyOf<T>::type;
        size_t s = 0;
        s += sizeof(T) * JB * JB;       // L11 (column-major, ld JB)
        s += sizeof(T) * (size_t)JB * cw; // U12 chunk (row-major, ld cw)
        s += sizeof(T) * 2 * NW * JB;   // candidate rows
        s += sizeof(K) * 2 * NW;        // candidate keys
        s += sizeof(int) * 2 * NW;      // candidate rows ids
        s += sizeof(int) * (size_t)R * NT; // src map
        s += sizeof(int) * 2 * JB;      // moved list
        s += sizeof(int) * (JB + 2);    // panel pivots, counter
        return (s + 15) & ~size_t(15);
    }
};

// Factor one m x n matrix with the whole CTA.  smem_raw must hold CtaLuSmem::bytes(cw, R);
// m <= R*NT.  Writes ipiv (1-based, PIVOT only) and *info_out.  Called by all threads.
template <typename T, int NT, int R, int JB, int TN, bool PIVOT>
__device__ __forceinline__ void getrf_cta_dev(int m, int n, T* a, int lda, int* piv_out,
                                              int* info_out, int cw, unsigned char* smem_raw)
{
    using K = typename KeyOf<T>::type;
    constexpr int NW = NT / 32;
    T* sL11 = reinterpret_cast<T*>(smem_raw);
    T* sU = sL11 + JB * JB;
    T* cand = sU + (size_t)JB * cw; // [2][NW][JB]
    K* ckey = reinterpret_cast<K*>(cand + 2 * NW * JB);
    int* crow = reinterpret_cast<int*>(ckey + 2 * NW);
    int* srcmap = crow + 2 * NW;
    int* moved = srcmap + R * NT;
    int* spiv = moved + 2 * JB;
    int* nmoved = spiv + JB;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mn = min(m, n);
    int inf = 0;

    T pv[R][JB];
    int lrow[R];

    for(int j0 = 0; j0 < mn; j0 += JB)
    {
        const int jb = min(JB, mn - j0);
        const int mp = m - j0;
        // ---- load the panel (rows j0..m-1, columns j0..j0+jb-1)
#pragma unroll
        for(int q = 0; q < R; ++q)
        {
            const int r = tid + q * NT;
            lrow[q] = r;
#pragma unroll
            for(int c = 0; c < JB; ++c)
                pv[q][c] = (r < mp && c < jb) ? a[ix(j0 + r, j0 + c, lda)] : T(0);
        }
        // ---- factor the panel, one barrier per column
#pragma unroll
        for(int c = 0; c < JB; ++c)
        {
            if(c < jb)
            {
                const int buf = c & 1;
                T* cb = cand + (size_t)buf * NW * JB;
                int prow = c, gw = 0;
                if(PIVOT)
                {
                    K bk = 0;
                    int br = INT_MAX;
                    bool any = false;
#pragma unroll
                    for(int q = 0; q < R; ++q)
                    {
                        const int r = tid + q * NT;
                        if(r < mp && lrow[q] >= c)
                        {
                            K kq = pivot_key(pv[q][c], lrow[q] == c);
                            if(!any || kq > bk || (kq == bk && lrow[q] < br))
                            {
                                bk = kq;
                                br = lrow[q];
                                any = true;
                            }
                        }
                    }
                    K wk;
                    const int wr = warp_argmax(bk, br, any, &wk);
                    if(any && br == wr)
                    {
#pragma unroll
                        for(int q = 0; q < R; ++q)
                            if(lrow[q] == wr && tid + q * NT < mp)
                            {
#pragma unroll
                                for(int cc = 0; cc < JB; ++cc)
                                    if(cc >= c)
                                        cb[warp * JB + cc] = pv[q][cc];
                            }
                    }
                    if(lane == 0)
                    {
                        ckey[buf * NW + warp] = wk;
                        crow[buf * NW + warp] = wr;
                    }
                    __syncthreads();
                    K gk = 0;
                    int gr = INT_MAX;
                    gw = -1;
#pragma unroll
                    for(int w = 0; w < NW; ++w)
                    {
                        const int rr = crow[buf * NW + w];
                        const K kw = ckey[buf * NW + w];
                        if(rr != INT_MAX && (gw < 0 || kw > gk || (kw == gk && rr < gr)))
                        {
                            gk = kw;
                            gr = rr;
                            gw = w;
                        }
                    }
                    prow = gr;
                }
                else
                {
#pragma unroll
                    for(int q = 0; q < R; ++q)
                        if(lrow[q] == c && tid + q * NT < mp)
                        {
#pragma unroll
                            for(int cc = 0; cc < JB; ++cc)
                                if(cc >= c)
                                    cb[cc] = pv[q][cc];
                        }
                    __syncthreads();
                }
                const T* prowv = cb + gw * JB;
                const T pivv = prowv[c];
                if(tid == 0)
                    spiv[c] = prow;
                if(pivv == T(0) && inf == 0)
                    inf = j0 + c + 1;
                Scaler<T> s;
                s.init(pivv);
#pragma unroll
                for(int q = 0; q < R; ++q)
                {
                    if(PIVOT)
                    {
                        if(lrow[q] == prow)
                            lrow[q] = c;
                        else if(lrow[q] == c)
                            lrow[q] = prow;
                    }
                    if(tid + q * NT < mp && lrow[q] > c)
                    {
                        const T l = s.apply(pv[q][c]);
                        pv[q][c] = l;
#pragma unroll
                        for(int cc = 0; cc < JB; ++cc)
                            if(cc > c)
                                pv[q][cc] = fma(-l, prowv[cc], pv[q][cc]);
                    }
                }
            }
        }
        // ---- write the panel back at its final row positions; L11 to shared memory
#pragma unroll
        for(int q = 0; q < R; ++q)
        {
            const int r = tid + q * NT;
            if(r < mp)
            {
#pragma unroll
                for(int cc = 0; cc < JB; ++cc)
                    if(cc < jb)
                        a[ix(j0 + lrow[q], j0 + cc, lda)] = pv[q][cc];
                if(lrow[q] < jb)
                {
#pragma unroll
                    for(int cc = 0; cc < JB; ++cc)
                        sL11[cc * JB + lrow[q]] = pv[q][cc];
                }
                srcmap[lrow[q]] = r;
            }
        }
        if(tid == 0)
            *nmoved = 0;
        __syncthreads();
        if(PIVOT)
        {
            if(tid < jb)
                piv_out[j0 + tid] = j0 + spiv[tid] + 1;
            // ---- list of moved rows (positions whose content changed)
            for(int p = tid; p < mp; p += NT)
                if(srcmap[p] != p)
                    moved[atomicAdd(nmoved, 1)] = p;
            __syncthreads();
            const int nm = *nmoved;
            // ---- apply the interchanges to the columns outside the panel, whole columns
            // per round so that no round reads a row a previous round already overwrote
            const int nother = n - jb;
            if(nm > 0 && nother > 0)
            {
                constexpr int KV = 8;
                const int cols_per_round = max(1, (NT * KV) / nm);
                for(int cb0 = 0; cb0 < nother; cb0 += cols_per_round)
                {
                    const int ncr = min(cols_per_round, nother - cb0);
                    const int npairs = ncr * nm;
                    T val[KV];
#pragma unroll
                    for(int v = 0; v < KV; ++v)
                    {
                        const int p = tid + v * NT;
                        if(p < npairs)
                        {
                            const int oc = cb0 + p / nm;
                            const int col = oc < j0 ? oc : oc + jb;
                            val[v] = a[ix(j0 + srcmap[moved[p % nm]], col, lda)];
                        }
                    }
                    __syncthreads();
#pragma unroll
                    for(int v = 0; v < KV; ++v)
                    {
                        const int p = tid + v * NT;
                        if(p < npairs)
                        {
                            const int oc = cb0 + p / nm;
                            const int col = oc < j0 ? oc : oc + jb;
                            a[ix(j0 + moved[p % nm], col, lda)] = val[v];
                        }
                    }
                    __syncthreads();
                }
            }
        }
        // ---- trailing update, column chunk by column chunk
        for(int c0 = j0 + jb; c0 < n; c0 += cw)
        {
            const int ncol = min(cw, n - c0);
            // U12 = L11^{-1} A12: one thread per column (reference dtrsm order L,L,N,U)
            for(int col = tid; col < ncol; col += NT)
            {
                T u[JB];
#pragma unroll
                for(int k = 0; k < JB; ++k)
                    u[k] = k < jb ? a[ix(j0 + k, c0 + col, lda)] : T(0);
#pragma unroll
                for(int k = 0; k < JB; ++k)
                {
#pragma unroll
                    for(int i = 0; i < JB; ++i)
                        if(i > k && i < jb)
                            u[i] = fma(-sL11[k * JB + i], u[k], u[i]);
                }
#pragma unroll
                for(int k = 0; k < JB; ++k)
                    if(k < jb)
                    {
                        a[ix(j0 + k, c0 + col, lda)] = u[k];
                        sU[(size_t)k * cw + col] = u[k];
                    }
            }
            __syncthreads();
            // A22 -= L21 * U12 for this chunk; each thread updates its own L21 rows
            for(int t0 = 0; t0 < ncol; t0 += TN)
            {
                T acc[R][TN];
#pragma unroll
                for(int q = 0; q < R; ++q)
                {
                    const bool mine = (tid + q * NT < mp) && lrow[q] >= jb;
#pragma unroll
                    for(int t = 0; t < TN; ++t)
                        acc[q][t] = (mine && t0 + t < ncol)
                                        ? a[ix(j0 + lrow[q], c0 + t0 + t, lda)]
                                        : T(0);
                }
#pragma unroll
                for(int k = 0; k < JB; ++k)
                {
                    if(k < jb)
                    {
                        T uk[TN];
#pragma unroll
                        for(int t = 0; t < TN; ++t)
                            uk[t] = sU[(size_t)k * cw + t0 + t];
#pragma unroll
                        for(int q = 0; q < R; ++q)
#pragma unroll
                            for(int t = 0; t < TN; ++t)
                                acc[q][t] = fma(-pv[q][k], uk[t], acc[q][t]);
                    }
                }
#pragma unroll
                for(int q = 0; q < R; ++q)
                {
                    const bool mine = (tid + q * NT < mp) && lrow[q] >= jb;
                    if(mine)
                    {
#pragma unroll
                        for(int t = 0; t < TN; ++t)
                            if(t0 + t < ncol)
                                a[ix(j0 + lrow[q], c0 + t0 + t, lda)] = acc[q][t];
                    }
                }
            }
            __syncthreads();
        }
    }
    if(tid == 0)
        *info_out = inf;
}

template <typename T, int NT, int R, int JB, int TN, bool PIVOT>
__global__ void __launch_bounds__(NT)
    getrf_cta_kernel(int m, int n, Batch<T> A, int lda, int* ipiv, int64_t strideP, int* info,
                     int cw, Gate gate)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int64_t b = blockIdx.x;
    if(gate.skip(b))
        return;
    getrf_cta_dev<T, NT, R, JB, TN, PIVOT>(m, n, A.at(b), lda, PIVOT ? ipiv + b * strideP : nullptr,
                                           info + b, cw, smem_raw);
}

} // namespace rsb
