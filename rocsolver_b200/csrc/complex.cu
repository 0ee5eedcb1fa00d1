// complex.cu -- the complex precisions (c = rocblas_float_complex, z = rocblas_double_complex)
// of the factor-and-solve path: getrf (and npvt), getrs (N, T, C), gesv, potrf, potrs, posv.
//
// The reference instantiates every hot-path routine for s, d, c and z
// (library/src/specialized/*_{s,d,c,z}.cpp); complex adds the conjugated solves
// (specialized/roclapack_trsm_specialized_kernels.hpp:219-380 conj_forward/backward
// substitution) and Hermitian Cholesky (roclapack_potf2.hpp:185-248 with conjugated dots).
//
// Design.  getrf: m, n <= 32 one warp per member with rows in registers
// (cgetrf_warp_kernel); m, n <= 64 one CTA per member with the member in registers, warps
// over column groups (cgetrf_reg_kernel); other members up to 96 KB one CTA per member
// factoring a shared-memory copy (cgetrf_smem_kernel); larger members the same device code
// in place in global memory (cgetrf_kernel).  Per column: the pivot is the first largest |re| + |im| (LAPACK izamax; a
// NaN only wins in the first position, through the same pivot keys as the real kernels), rows
// are interchanged over all columns, the column is scaled by the reciprocal (|pivot| >=
// sfmin) or by division, and the trailing matrix takes the rank-1 update.  potrf: the same
// shared-memory / global split.  getrs and potrs for n <= 256: one warp per member and
// right-hand side, no block barriers (cgetrs_warp_kernel, cpotrs_warp_kernel); larger n one
// CTA per member sweeping one unknown at a time.
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

// larger components between which |z|^2 neither overflows nor underflows
template <typename R>
struct CxSafe;
template <>
struct CxSafe<double>
{
    static __device__ __forceinline__ double lo() { return 0x1p-500; }
    static __device__ __forceinline__ double hi() { return 0x1p+500; }
};
template <>
struct CxSafe<float>
{
    static __device__ __forceinline__ float lo() { return 0x1p-60f; }
    static __device__ __forceinline__ float hi() { return 0x1p+60f; }
};

// |z| >= sfmin (LAPACK zgetf2's test on the pivot's modulus): the larger component decides
// it without a square root unless z is tiny
template <typename C>
__device__ __forceinline__ bool cbig(C z)
{
    using R = typename CxReal<C>::R;
    return fmax(fabs(z.x), fabs(z.y)) >= Lim<R>::sfmin() || hypot(z.x, z.y) >= Lim<R>::sfmin();
}

// 1 / z for |z| >= sfmin with one real reciprocal: 1/z = conj(z) / |z|^2 while the larger
// component lies in the safe range; otherwise z is first scaled by the power of two 2^-e of
// its larger component (exact), 1/z = conj(z') / |z'|^2 * 2^-e
template <typename C>
__device__ __forceinline__ C crcp(C z)
{
    using R = typename CxReal<C>::R;
    const R mx = fmax(fabs(z.x), fabs(z.y));
    if(mx >= CxSafe<R>::lo() && mx <= CxSafe<R>::hi())
    {
        const R inv = Lim<R>::rcp(z.x * z.x + z.y * z.y);
        return cx<C>(z.x * inv, -z.y * inv);
    }
    const int e = ilogb(mx);
    const R x = scalbn(z.x, -e), y = scalbn(z.y, -e);
    const R inv = R(1) / (x * x + y * y);
    return cx<C>(scalbn(x * inv, -e), scalbn(-y * inv, -e));
}

// pivot-search records of one column, double-buffered by column parity so that the next
// column's records never overwrite ones still being read
template <typename C>
struct CxPivRec
{
    using K = typename KeyOf<typename CxReal<C>::R>::type;
    K key[2][CPX_NT / 32];
    int row[2][CPX_NT / 32];
    C val[2][CPX_NT / 32];
    C ajj[2];
};

// LU of one m x n member at a (leading dimension lda: global memory, or the member's copy in
// shared memory) by the whole CTA; writes ipiv (PIVOT) and returns info.  Per column, three
// barriers: (1) the pivot search over the rows (threads over rows; each warp's winner
// publishes its key, row and value, thread 0 the diagonal entry), (2) the interchange of the
// other columns, together with the scaling of the column below the diagonal (the pivot row's
// slot takes the old diagonal entry), (3) the rank-1 update of the trailing matrix with warps
// over columns and lanes over rows (consecutive rows of a column are contiguous: coalesced in
// global memory, conflict-free rows in shared memory).
template <typename C, bool PIVOT>
__device__ __forceinline__ int cgetrf_dev(int m, int n, C* a, int lda, int* piv,
                                          CxPivRec<C>& rec)
{
    using R = typename CxReal<C>::R;
    using K = typename KeyOf<R>::type;
    constexpr int NW = CPX_NT / 32;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mn = min(m, n);
    int inf = 0;
    for(int j = 0; j < mn; ++j)
    {
        const int buf = j & 1;
        // ---- (1) pivot search: this thread's first largest |re| + |im| among its rows
        const int rend = PIVOT ? m : j + 1; // rows searched: j .. rend-1
        if(j + warp * 32 >= rend)
        {
            // no candidate row in this warp (for any of its strided passes when m > NT the
            // first pass already has one)
            if(lane == 0)
                rec.row[buf][warp] = INT_MAX;
        }
        else
        {
            K bk = 0;
            int br = INT_MAX;
            C bv = cx<C>(0, 0);
            for(int i = j + tid; i < rend; i += CPX_NT)
            {
                const C v = RSB_AT(a, i, j, lda, m, n);
                if(i == j)
                    rec.ajj[buf] = v;
                const K k = pivot_key((R)(fabs(v.x) + fabs(v.y)), i == j);
                if(br == INT_MAX || k > bk)
                {
                    bk = k;
                    br = i;
                    bv = v;
                }
            }
            K wk;
            const int wr = warp_argmax(bk, br, br != INT_MAX, &wk);
            if(br == wr && br != INT_MAX)
            {
                rec.key[buf][warp] = wk;
                rec.row[buf][warp] = wr;
                rec.val[buf][warp] = bv;
            }
        }
        __syncthreads();
        const bool rv = lane < NW && rec.row[buf][lane] != INT_MAX;
        K gk;
        const int p = warp_argmax(rv ? rec.key[buf][lane] : K(0),
                                  rv ? rec.row[buf][lane] : INT_MAX, rv, &gk);
        const int gw = __ffs(__ballot_sync(0xffffffffu, rv && rec.row[buf][lane] == p)) - 1;
        const C pv = rec.val[buf][gw];
        const C ajj = rec.ajj[buf];
        if(PIVOT && tid == 0)
            piv[j] = p + 1;
        // ---- (2) interchange rows j and p outside column j; scale column j below the pivot
        if(!czero(pv))
        {
            if(p != j && tid < n)
                for(int c = tid; c < n; c += CPX_NT)
                    if(c != j)
                    {
                        const C t = RSB_AT(a, j, c, lda, m, n);
                        RSB_AT(a, j, c, lda, m, n) = RSB_AT(a, p, c, lda, m, n);
                        RSB_AT(a, p, c, lda, m, n) = t;
                    }
            if(j + 1 + tid < m) // only threads with a row to scale form the reciprocal
            {
                const bool recip = cbig(pv);
                const C r = recip ? crcp(pv) : pv;
                for(int i = j + 1 + tid; i < m; i += CPX_NT)
                {
                    C& e = RSB_AT(a, i, j, lda, m, n);
                    e = recip ? cmul(i == p ? ajj : e, r) : cdiv(i == p ? ajj : e, pv);
                }
            }
            if(tid == 0)
                RSB_AT(a, j, j, lda, m, n) = pv;
        }
        else if(inf == 0)
            inf = j + 1;
        __syncthreads();
        // ---- (3) A(j+1:m, j+1:n) -= A(j+1:m, j) A(j, j+1:n)
        for(int c = j + 1 + warp; c < n; c += NW)
        {
            const C u = RSB_AT(a, j, c, lda, m, n);
            if(czero(u))
                continue;
            for(int i = j + 1 + lane; i < m; i += 32)
            {
                C& t = RSB_AT(a, i, c, lda, m, n);
                t = csub(t, cmul(RSB_AT(a, i, j, lda, m, n), u));
            }
        }
        __syncthreads();
    }
    return inf;
}

template <typename C, bool PIVOT>
__global__ void __launch_bounds__(CPX_NT)
    cgetrf_kernel(int m, int n, Batch<C> A, int lda, int* ipiv, int64_t strideP, int* info,
                  Gate gate)
{
    __shared__ CxPivRec<C> rec;
    const int64_t b = blockIdx.x;
    if(gate.skip(b))
        return;
    const int inf = cgetrf_dev<C, PIVOT>(m, n, A.at(b), lda, PIVOT ? ipiv + b * strideP : nullptr,
                                         rec);
    if(threadIdx.x == 0)
        info[b] = inf;
}

// ---- m, n <= NMAX <= 32: one warp per member, lane i holds row i in registers (the real
// getrf_warp_kernel's scheme).  Per column: every lane forms the reciprocal of its own
// candidate while the warp reduction runs, the winner publishes its row (and reciprocal)
// through a double-buffered shared-memory row ordered by __syncwarp, rows are relabelled
// instead of moved, and each lane updates its own row.
constexpr int CPX_WPB = 4; // members (warps) per CTA

template <typename C, int NMAX, bool PIVOT>
__global__ void __launch_bounds__(32 * CPX_WPB)
    cgetrf_warp_kernel(int m, int n, Batch<C> A, int lda, int* ipiv, int64_t strideP,
                       int* info, int bc, Gate gate)
{
    using R = typename CxReal<C>::R;
    __shared__ C srow[CPX_WPB][2][NMAX + 1]; // pivot row; element NMAX: its reciprocal
    __shared__ int sbig[CPX_WPB][2];         // |pivot| >= sfmin
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t b = (int64_t)blockIdx.x * CPX_WPB + warp;
    if(b >= bc || gate.skip(b))
        return;
    C* a = A.at(b);
    C r[NMAX];
#pragma unroll
    for(int j = 0; j < NMAX; ++j)
        r[j] = (lane < m && j < n) ? RSB_AT(a, lane, j, lda, m, n) : cx<C>(0, 0);
    int myrow = lane, mypiv = lane + 1, inf = 0;
    const int mn = min(m, n);
#pragma unroll
    for(int k = 0; k < NMAX; ++k)
    {
        if(k < mn)
        {
        const int buf = k & 1;
        C* row = srow[warp][buf];
        // this lane's candidate: its reciprocal (used if it wins) formed off the serial path
        const C x0 = r[k];
        const bool big = cbig(x0);
        const C rc = big ? crcp(x0) : x0;
        int prow = k;
        if(PIVOT)
            prow = warp_argmax_fast(pivot_key((R)(fabs(x0.x) + fabs(x0.y)), myrow == k), myrow,
                                    lane < m && myrow >= k);
        if(myrow == prow)
        {
#pragma unroll
            for(int j = k; j < NMAX; ++j)
                row[j] = r[j];
            row[NMAX] = rc;
            sbig[warp][buf] = big;
        }
        __syncwarp();
        const C piv = row[k];
        const C rcp = row[NMAX];
        const bool pbig = sbig[warp][buf] != 0;
        if(lane == k)
            mypiv = prow + 1;
        if(czero(piv) && inf == 0)
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
            // LAPACK zgetf2: multiply by the reciprocal when |pivot| >= sfmin, else divide;
            // a zero pivot leaves the column unscaled
            C l = r[k];
            if(!czero(piv))
                l = pbig ? cmul(l, rcp) : cdiv(l, piv);
            r[k] = l;
#pragma unroll
            for(int j = k + 1; j < NMAX; ++j)
                r[j] = csub(r[j], cmul(l, row[j]));
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

template <typename C, int NMAX>
static rocblas_status cx_getrf_warp(cudaStream_t s, int m, int n, Batch<C> A, int lda,
                                    int* ipiv, int64_t sP, int* info, int bc, bool pivot, Gate g)
{
    const unsigned grid = (unsigned)((bc + CPX_WPB - 1) / CPX_WPB);
    if(pivot)
        cgetrf_warp_kernel<C, NMAX, true><<<grid, 32 * CPX_WPB, 0, s>>>(m, n, A, lda, ipiv, sP,
                                                                        info, bc, g);
    else
        cgetrf_warp_kernel<C, NMAX, false><<<grid, 32 * CPX_WPB, 0, s>>>(m, n, A, lda, ipiv, sP,
                                                                         info, bc, g);
    return cudaGetLastError() == cudaSuccess ? rocblas_status_success
                                             : rocblas_status_internal_error;
}

// ---- m, n <= 64, not both <= 32: one CTA per member, the whole member in registers.  Warp g
// holds columns g*NC .. g*NC+NC-1 and lane i rows i and i+32 (S slots).  Rows stay where they
// are and are relabelled (myrow = the row's current position), as in the warp kernel.  Per
// column k one CTA barrier: before it the warp holding column k searches it, scales it by the
// pivot's reciprocal and publishes the multipliers and the pivot (double-buffered by the
// parity of k); after it every warp right of the column takes the pivot row's part of its own
// columns from the pivot lane (warp-private shared memory, ordered by __syncwarp) and updates
// its rows, and the warp holding column k+1 searches that next.
template <typename C>
struct CxRegPiv
{
    C pv;
    int slot, label;
};

// search, pivot and scale column kc of the calling warp: v[s] holds the column's entry of row
// lane + 32 s and takes its multiplier; the multipliers go to col (by slot), the pivot to pr
template <typename C, int S, bool PIVOT>
__device__ __forceinline__ void cx_reg_pivot(int kc, int m, C (&v)[S], const int (&myrow)[S],
                                             CxRegPiv<C>& pr, C* col, int* piv)
{
    using R = typename CxReal<C>::R;
    using K = typename KeyOf<R>::type;
    const int lane = threadIdx.x & 31;
    K bk = 0;
    int bl = INT_MAX, bs = 0;
#pragma unroll
    for(int s = 0; s < S; ++s)
    {
        const bool ok = lane + 32 * s < m && (PIVOT ? myrow[s] >= kc : myrow[s] == kc);
        const K key = pivot_key((R)(fabs(v[s].x) + fabs(v[s].y)), myrow[s] == kc);
        if(ok && (bl == INT_MAX || key > bk || (key == bk && myrow[s] < bl)))
        {
            bk = key;
            bl = myrow[s];
            bs = s;
        }
    }
    const int p = warp_argmax_fast(bk, bl, bl != INT_MAX); // row kc is always a candidate
    if(bl == p)
    {
        pr.pv = bs == 0 ? v[0] : v[S - 1];
        pr.slot = lane + 32 * bs;
        pr.label = p;
        if(PIVOT)
            piv[kc] = p + 1;
    }
    __syncwarp();
    // every lane forms the same reciprocal of the broadcast pivot
    const C pv = pr.pv;
    const bool pb = cbig(pv);
    const C r = pb ? crcp(pv) : pv;
    const int slot = pr.slot;
#pragma unroll
    for(int s = 0; s < S; ++s)
        if(lane + 32 * s < m && myrow[s] >= kc && lane + 32 * s != slot)
        {
            // LAPACK zgetf2: reciprocal when |pivot| >= sfmin, else division; a zero pivot
            // leaves the column unscaled
            C l = v[s];
            if(!czero(pv))
                l = pb ? cmul(l, r) : cdiv(l, pv);
            v[s] = l;
            col[lane + 32 * s] = l;
        }
}

// complex float members fit three CTAs per SM (80 registers), complex double two
template <typename C, int NC, int S, bool PIVOT>
__global__ void __launch_bounds__(32 * (64 / NC), sizeof(C) == 8 ? 3 : 2)
    cgetrf_reg_kernel(int m, int n, Batch<C> A, int lda, int* ipiv, int64_t strideP, int* info,
                      Gate gate)
{
    constexpr int G = 64 / NC;
    __shared__ CxRegPiv<C> spiv[2];
    __shared__ C scol[2][32 * S];
    __shared__ C sprow[G][NC];
    const int64_t b = blockIdx.x;
    if(gate.skip(b))
        return;
    C* a = A.at(b);
    int* piv = PIVOT ? ipiv + b * strideP : nullptr;
    const int g = threadIdx.x >> 5, lane = threadIdx.x & 31;
    C r[S][NC];
    int myrow[S];
#pragma unroll
    for(int s = 0; s < S; ++s)
    {
        myrow[s] = lane + 32 * s;
#pragma unroll
        for(int j = 0; j < NC; ++j)
            r[s][j] = (lane + 32 * s < m && g * NC + j < n)
                          ? RSB_AT(a, lane + 32 * s, g * NC + j, lda, m, n)
                          : cx<C>(0, 0);
    }
    const int mn = min(m, n);
    int inf = 0;
    if(g == 0)
    {
        C v[S];
#pragma unroll
        for(int s = 0; s < S; ++s)
            v[s] = r[s][0];
        cx_reg_pivot<C, S, PIVOT>(0, m, v, myrow, spiv[0], scol[0], piv);
#pragma unroll
        for(int s = 0; s < S; ++s)
            r[s][0] = v[s];
    }
    const int ng = (mn + NC - 1) / NC;
    for(int g0 = 0; g0 < ng; ++g0)
    {
#pragma unroll
        for(int kk = 0; kk < NC; ++kk)
        {
            const int k = g0 * NC + kk;
            if(k < mn)
            {
                const int buf = k & 1;
                __syncthreads();
                const int ps = spiv[buf].slot, p = spiv[buf].label;
                if(inf == 0 && czero(spiv[buf].pv))
                    inf = k + 1;
                if(PIVOT)
#pragma unroll
                    for(int s = 0; s < S; ++s)
                        myrow[s] = myrow[s] == p ? k : (myrow[s] == k ? p : myrow[s]);
                if(g >= g0)
                {
                    // the pivot row's part of this warp's columns right of k
                    if(lane == (ps & 31))
                    {
#pragma unroll
                        for(int j = 0; j < NC; ++j)
                            if(g > g0 || j > kk)
                                sprow[g][j] = (S == 1 || ps < 32) ? r[0][j] : r[S - 1][j];
                    }
                    __syncwarp();
                    C l[S];
                    bool act[S];
#pragma unroll
                    for(int s = 0; s < S; ++s)
                    {
                        act[s] = lane + 32 * s < m && myrow[s] > k;
                        l[s] = act[s] ? scol[buf][lane + 32 * s] : cx<C>(0, 0);
                    }
                    if(g == g0)
                    {
#pragma unroll
                        for(int j = kk + 1; j < NC; ++j)
                        {
                            const C u = sprow[g][j];
#pragma unroll
                            for(int s = 0; s < S; ++s)
                                if(act[s])
                                    r[s][j] = csub(r[s][j], cmul(l[s], u));
                        }
                    }
                    else
                    {
#pragma unroll
                        for(int j = 0; j < NC; ++j)
                        {
                            const C u = sprow[g][j];
#pragma unroll
                            for(int s = 0; s < S; ++s)
                                if(act[s])
                                    r[s][j] = csub(r[s][j], cmul(l[s], u));
                        }
                    }
                }
                // the next column's pivot, by the warp that holds it
                if(k + 1 < mn)
                {
                    const int jn = (kk + 1) % NC;
                    if(kk + 1 < NC ? g == g0 : g == g0 + 1)
                    {
                        C v[S];
#pragma unroll
                        for(int s = 0; s < S; ++s)
                            v[s] = r[s][jn];
                        cx_reg_pivot<C, S, PIVOT>(k + 1, m, v, myrow, spiv[buf ^ 1],
                                                  scol[buf ^ 1], piv);
#pragma unroll
                        for(int s = 0; s < S; ++s)
                            r[s][jn] = v[s];
                    }
                }
            }
        }
    }
#pragma unroll
    for(int s = 0; s < S; ++s)
        if(lane + 32 * s < m)
#pragma unroll
            for(int j = 0; j < NC; ++j)
                if(g * NC + j < n)
                    RSB_AT(a, myrow[s], g * NC + j, lda, m, n) = r[s][j];
    if(threadIdx.x == 0)
        info[b] = inf;
}

template <typename C, int NC>
static rocblas_status cx_getrf_reg(cudaStream_t s, int m, int n, Batch<C> A, int lda,
                                   int* ipiv, int64_t sP, int* info, int bc, bool pivot, Gate g)
{
    constexpr int NT = 32 * (64 / NC);
    if(m > 32)
    {
        if(pivot)
            cgetrf_reg_kernel<C, NC, 2, true><<<bc, NT, 0, s>>>(m, n, A, lda, ipiv, sP, info, g);
        else
            cgetrf_reg_kernel<C, NC, 2, false><<<bc, NT, 0, s>>>(m, n, A, lda, ipiv, sP, info, g);
    }
    else
    {
        if(pivot)
            cgetrf_reg_kernel<C, NC, 1, true><<<bc, NT, 0, s>>>(m, n, A, lda, ipiv, sP, info, g);
        else
            cgetrf_reg_kernel<C, NC, 1, false><<<bc, NT, 0, s>>>(m, n, A, lda, ipiv, sP, info, g);
    }
    return cudaGetLastError() == cudaSuccess ? rocblas_status_success
                                             : rocblas_status_internal_error;
}

// members of at most CPX_SMEM_MAX bytes are factored in shared memory (one copy in, one out)
constexpr int CPX_SMEM_MAX = 96 * 1024;

template <typename C, bool PIVOT>
__global__ void __launch_bounds__(CPX_NT)
    cgetrf_smem_kernel(int m, int n, Batch<C> A, int lda, int* ipiv, int64_t strideP, int* info,
                       Gate gate)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sa = reinterpret_cast<C*>(smem_raw); // m x n, leading dimension m
    __shared__ CxPivRec<C> rec;
    constexpr int NW = CPX_NT / 32;
    const int64_t b = blockIdx.x;
    if(gate.skip(b))
        return;
    C* a = A.at(b);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for(int c = warp; c < n; c += NW)
        for(int i = lane; i < m; i += 32)
            sa[i + (size_t)c * m] = RSB_AT(a, i, c, lda, m, n);
    __syncthreads();
    const int inf = cgetrf_dev<C, PIVOT>(m, n, sa, m, PIVOT ? ipiv + b * strideP : nullptr, rec);
    for(int c = warp; c < n; c += NW)
        for(int i = lane; i < m; i += 32)
            RSB_AT(a, i, c, lda, m, n) = sa[i + (size_t)c * m];
    if(threadIdx.x == 0)
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

// Hermitian Cholesky of one member at a (global memory, or its copy in shared memory),
// right-looking: A = L L^H (lower) or U^H U (upper); returns info = first order whose pivot
// real(a_jj) - sum |l_jk|^2 is <= 0 or NaN (that value is stored in a_jj, then the
// factorisation stops, as LAPACK zpotf2 does).  The other triangle is not touched.  The
// trailing update runs with warps over columns and lanes over rows.
template <typename C>
__device__ __forceinline__ int cpotrf_dev(int upper, int n, C* a, int lda)
{
    using R = typename CxReal<C>::R;
    constexpr int NW = CPX_NT / 32;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for(int j = 0; j < n; ++j)
    {
        const R ajj = RSB_AT(a, j, j, lda, n, n).x;
        __syncthreads();
        if(ajj <= R(0) || isnan(ajj))
        {
            if(tid == 0)
                RSB_AT(a, j, j, lda, n, n) = cx<C>(ajj, 0);
            __syncthreads();
            return j + 1;
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
        // trailing Hermitian update of the referenced triangle, column k by one warp
        for(int k = j + 1 + warp; k < n; k += NW)
        {
            if(!upper) // L(i,k) -= L(i,j) conj(L(k,j)), i >= k
            {
                const C lk = cconj(RSB_AT(a, k, j, lda, n, n));
                for(int i = k + lane; i < n; i += 32)
                {
                    C& v = RSB_AT(a, i, k, lda, n, n);
                    v = csub(v, cmul(RSB_AT(a, i, j, lda, n, n), lk));
                }
            }
            else // U(i,k) -= conj(U(j,i)) U(j,k), j < i <= k
            {
                const C uk = RSB_AT(a, j, k, lda, n, n);
                for(int i = j + 1 + lane; i <= k; i += 32)
                {
                    C& v = RSB_AT(a, i, k, lda, n, n);
                    v = csub(v, cmul(cconj(RSB_AT(a, j, i, lda, n, n)), uk));
                }
            }
        }
        __syncthreads();
    }
    return 0;
}

template <typename C>
__global__ void __launch_bounds__(CPX_NT)
    cpotrf_kernel(int upper, int n, Batch<C> A, int lda, int* info)
{
    const int inf = cpotrf_dev<C>(upper, n, A.at(blockIdx.x), lda);
    if(threadIdx.x == 0)
        info[blockIdx.x] = inf;
}

// members of at most CPX_SMEM_MAX bytes: the referenced triangle is factored in shared memory
// (larger members run cpotrf_kernel in place: after a failure their trailing part holds the
// updates of the finished columns, as LAPACK's blocked zpotrf leaves its trailing blocks)
template <typename C>
__global__ void __launch_bounds__(CPX_NT)
    cpotrf_smem_kernel(int upper, int n, Batch<C> A, int lda, int* info)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sa = reinterpret_cast<C*>(smem_raw); // n x n, leading dimension n
    constexpr int NW = CPX_NT / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    C* a = A.at(blockIdx.x);
    for(int c = warp; c < n; c += NW)
        for(int i = upper ? lane : c + lane; i < (upper ? c + 1 : n); i += 32)
            sa[i + (size_t)c * n] = RSB_AT(a, i, c, lda, n, n);
    __syncthreads();
    const int inf = cpotrf_dev<C>(upper, n, sa, n);
    // write back what LAPACK zpotf2 leaves: everything, or after a failure at order k the
    // finished columns (rows, for upper) before k and the failing pivot; the trailing part,
    // updated here but not by zpotf2, keeps its input
    const int k = inf ? inf - 1 : n;
    for(int c = warp; c < n; c += NW)
        for(int i = upper ? lane : c + lane; i < (upper ? c + 1 : n); i += 32)
            if(min(i, c) < k || (i == k && c == k))
                RSB_AT(a, i, c, lda, n, n) = sa[i + (size_t)c * n];
    if(threadIdx.x == 0)
        info[blockIdx.x] = inf;
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

// ---- warp-per-right-hand-side solves (n <= 32 * Q): lane l holds rows l, l + 32, ... of
// the vector in registers; no block barriers.  Two sweep forms, chosen so that the lanes read
// contiguous memory: AXPY (column-oriented: once x_k is final, the rows on the far side of k
// take T(i,k) x_k, lanes over i) and DOT (row-oriented: x_i = (x_i - sum_k T(i,k) x_k) /
// T(i,i), lanes over k, one warp reduction per row).  get(i, k) returns the element T(i, k)
// of the triangular matrix (conjugated by the caller when the solve needs it); FWD solves
// rows in increasing order (T lower), else decreasing (T upper); UNIT skips the diagonal.
template <typename C>
__device__ __forceinline__ C cshfl(C v, int src)
{
    return cx<C>(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
template <typename C>
__device__ __forceinline__ C cshfl_xor(C v, int m)
{
    return cx<C>(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

template <typename C, int Q, bool FWD, bool AXPY, bool UNIT, typename Get>
__device__ __forceinline__ void warp_trsv(int n, C (&x)[Q], Get get)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for(int qs = 0; qs < Q; ++qs)
    {
        const int q0 = FWD ? qs : Q - 1 - qs; // register holding the sequential index
        for(int ks = 0; ks < 32; ++ks)
        {
            const int kk = FWD ? ks : 31 - ks;
            const int k = 32 * q0 + kk; // the row (DOT) or column (AXPY) being finished
            if(k >= n)
            {
                if(FWD)
                    break;
                continue;
            }
            if(AXPY)
            {
                if(!UNIT && lane == kk)
                    x[q0] = cdiv(x[q0], get(k, k));
                const C xk = cshfl(x[q0], kk);
#pragma unroll
                for(int q = 0; q < Q; ++q)
                {
                    const int i = lane + 32 * q;
                    if((FWD ? q >= q0 : q <= q0) && (FWD ? i > k : i < k) && i < n)
                        x[q] = csub(x[q], cmul(get(i, k), xk));
                }
            }
            else
            {
                C part = cx<C>(0, 0);
#pragma unroll
                for(int q = 0; q < Q; ++q)
                {
                    const int j = lane + 32 * q;
                    if((FWD ? q <= q0 : q >= q0) && (FWD ? j < k : j > k) && j < n)
                    {
                        const C t = cmul(get(k, j), x[q]);
                        part = cx<C>(part.x + t.x, part.y + t.y);
                    }
                }
#pragma unroll
                for(int m = 16; m >= 1; m >>= 1)
                {
                    const C o = cshfl_xor(part, m);
                    part = cx<C>(part.x + o.x, part.y + o.y);
                }
                if(lane == kk)
                {
                    const C v = csub(x[q0], part);
                    x[q0] = UNIT ? v : cdiv(v, get(k, k));
                }
            }
        }
    }
}

// source position of each of this lane's rows under the interchanges piv[0..n-1] applied in
// order (LAPACK laswp, incx = 1): position i holds original row src(i)
template <int Q>
__device__ __forceinline__ void warp_perm_src_q(const int* piv, int n, int (&src)[Q])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for(int q = 0; q < Q; ++q)
        src[q] = lane + 32 * q;
    for(int k = n - 1; k >= 0; --k)
    {
        const int p = piv[k] - 1;
        RSB_CHECK_PIV(piv[k], n, __LINE__);
#pragma unroll
        for(int q = 0; q < Q; ++q)
            src[q] = src[q] == k ? p : (src[q] == p ? k : src[q]);
    }
}

// getrs with one warp per (member, right-hand-side column); four warps per CTA
template <typename C, int Q>
__global__ void __launch_bounds__(128)
    cgetrs_warp_kernel(int trans, int n, int nrhs, Batch<C> A, int lda, const int* ipiv,
                       int64_t strideP, Batch<C> B, int ldb, const int* skip, Gate gate,
                       int64_t tasks)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t task = (int64_t)blockIdx.x * 4 + warp;
    if(task >= tasks)
        return;
    const int64_t b = task / nrhs;
    const int col = (int)(task % nrhs);
    if((skip && skip[b] != 0) || gate.skip(b))
        return;
    const C* a = A.at(b);
    C* xb = B.at(b);
    int src[Q];
    if(ipiv)
        warp_perm_src_q<Q>(ipiv + b * strideP, n, src);
    else
#pragma unroll
        for(int q = 0; q < Q; ++q)
            src[q] = lane + 32 * q;
    C x[Q];
    const bool cj = trans == 2;
#pragma unroll
    for(int q = 0; q < Q; ++q)
    {
        const int i = lane + 32 * q;
        x[q] = i < n ? RSB_AT(xb, trans == 0 ? src[q] : i, col, ldb, n, nrhs) : cx<C>(0, 0);
    }
    if(trans == 0)
    {
        // L y = P b (unit lower, columns of L), U x = y (columns of U)
        auto el = [&](int i, int k) { return RSB_AT(a, i, k, lda, n, n); };
        warp_trsv<C, Q, true, true, true>(n, x, el);
        warp_trsv<C, Q, false, true, false>(n, x, el);
    }
    else
    {
        // op(U)^T y = b: row i of U^T is column i of U (DOT, lanes over k); op(L)^T x = y
        auto opT = [&](int i, int k) {
            const C v = RSB_AT(a, k, i, lda, n, n);
            return cj ? cconj(v) : v;
        };
        warp_trsv<C, Q, true, false, false>(n, x, opT);
        warp_trsv<C, Q, false, false, true>(n, x, opT);
    }
    __syncwarp();
#pragma unroll
    for(int q = 0; q < Q; ++q)
    {
        const int i = lane + 32 * q;
        if(i < n)
            RSB_AT(xb, trans == 0 ? i : src[q], col, ldb, n, nrhs) = x[q];
    }
}

// potrs with one warp per (member, right-hand-side column): lower L L^H: L y = b (columns of
// L), L^H x = y (rows of L^H = conjugated columns of L, DOT); upper U^H U: U^H y = b (DOT on
// conjugated columns of U), U x = y (columns of U)
template <typename C, int Q>
__global__ void __launch_bounds__(128)
    cpotrs_warp_kernel(int upper, int n, int nrhs, Batch<C> A, int lda, Batch<C> B, int ldb,
                       const int* skip, int64_t tasks)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t task = (int64_t)blockIdx.x * 4 + warp;
    if(task >= tasks)
        return;
    const int64_t b = task / nrhs;
    const int col = (int)(task % nrhs);
    if(skip && skip[b] != 0)
        return;
    const C* a = A.at(b);
    C* xb = B.at(b);
    C x[Q];
#pragma unroll
    for(int q = 0; q < Q; ++q)
    {
        const int i = lane + 32 * q;
        x[q] = i < n ? RSB_AT(xb, i, col, ldb, n, nrhs) : cx<C>(0, 0);
    }
    auto el = [&](int i, int k) { return RSB_AT(a, i, k, lda, n, n); };
    auto elH = [&](int i, int k) { return cconj(RSB_AT(a, k, i, lda, n, n)); };
    if(upper)
    {
        warp_trsv<C, Q, true, false, false>(n, x, elH);
        warp_trsv<C, Q, false, true, false>(n, x, el);
    }
    else
    {
        warp_trsv<C, Q, true, true, false>(n, x, el);
        warp_trsv<C, Q, false, false, false>(n, x, elH);
    }
#pragma unroll
    for(int q = 0; q < Q; ++q)
    {
        const int i = lane + 32 * q;
        if(i < n)
            RSB_AT(xb, i, col, ldb, n, nrhs) = x[q];
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
    if(m <= 32 && n <= 32)
    {
        RSB_LOG_KERNEL("cgetrf_warp_kernel");
        const int mx = max(m, n);
        if(mx <= 8)
            return cx_getrf_warp<C, 8>(s, m, n, A, lda, ipiv, sP, info, bc, pivot, g);
        if(mx <= 16)
            return cx_getrf_warp<C, 16>(s, m, n, A, lda, ipiv, sP, info, bc, pivot, g);
        return cx_getrf_warp<C, 32>(s, m, n, A, lda, ipiv, sP, info, bc, pivot, g);
    }
    if(m <= 64 && n <= 64)
    {
        RSB_LOG_KERNEL("cgetrf_reg_kernel");
        return cx_getrf_reg<C, 8>(s, m, n, A, lda, ipiv, sP, info, bc, pivot, g);
    }
    const size_t bytes = sizeof(C) * (size_t)m * n;
    if(bytes <= CPX_SMEM_MAX)
    {
        RSB_LOG_KERNEL("cgetrf_smem_kernel");
        auto k = pivot ? cgetrf_smem_kernel<C, true> : cgetrf_smem_kernel<C, false>;
        if(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, CPX_SMEM_MAX)
           != cudaSuccess)
            return rocblas_status_internal_error;
        k<<<bc, CPX_NT, bytes, s>>>(m, n, A, lda, ipiv, sP, info, g);
        return status_of_launch();
    }
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
    if(n <= 256)
    {
        RSB_LOG_KERNEL("cgetrs_warp_kernel");
        const int64_t tasks = (int64_t)bc * nrhs;
        const unsigned grid = (unsigned)((tasks + 3) / 4);
        if(n <= 32)
            cgetrs_warp_kernel<C, 1><<<grid, 128, 0, s>>>(trans, n, nrhs, A, lda, ipiv, sP, B,
                                                          ldb, skip, g, tasks);
        else if(n <= 64)
            cgetrs_warp_kernel<C, 2><<<grid, 128, 0, s>>>(trans, n, nrhs, A, lda, ipiv, sP, B,
                                                          ldb, skip, g, tasks);
        else if(n <= 128)
            cgetrs_warp_kernel<C, 4><<<grid, 128, 0, s>>>(trans, n, nrhs, A, lda, ipiv, sP, B,
                                                          ldb, skip, g, tasks);
        else
            cgetrs_warp_kernel<C, 8><<<grid, 128, 0, s>>>(trans, n, nrhs, A, lda, ipiv, sP, B,
                                                          ldb, skip, g, tasks);
        return status_of_launch();
    }
    RSB_LOG_KERNEL("cgetrs_kernel");
    cgetrs_kernel<C><<<bc, CPX_NT, 0, s>>>(trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, g);
    return status_of_launch();
}
template <typename C>
rocblas_status cx_potrf(cudaStream_t s, int upper, int n, Batch<C> A, int lda, int* info, int bc)
{
    const size_t bytes = sizeof(C) * (size_t)n * n;
    if(bytes <= CPX_SMEM_MAX)
    {
        RSB_LOG_KERNEL("cpotrf_smem_kernel");
        if(cudaFuncSetAttribute(cpotrf_smem_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                CPX_SMEM_MAX)
           != cudaSuccess)
            return rocblas_status_internal_error;
        cpotrf_smem_kernel<C><<<bc, CPX_NT, bytes, s>>>(upper, n, A, lda, info);
        return status_of_launch();
    }
    RSB_LOG_KERNEL("cpotrf_kernel");
    cpotrf_kernel<C><<<bc, CPX_NT, 0, s>>>(upper, n, A, lda, info);
    return status_of_launch();
}
template <typename C>
rocblas_status cx_potrs(cudaStream_t s, int upper, int n, int nrhs, Batch<C> A, int lda,
                        Batch<C> B, int ldb, const int* skip, int bc)
{
    if(n <= 256)
    {
        RSB_LOG_KERNEL("cpotrs_warp_kernel");
        const int64_t tasks = (int64_t)bc * nrhs;
        const unsigned grid = (unsigned)((tasks + 3) / 4);
        if(n <= 32)
            cpotrs_warp_kernel<C, 1><<<grid, 128, 0, s>>>(upper, n, nrhs, A, lda, B, ldb, skip,
                                                          tasks);
        else if(n <= 64)
            cpotrs_warp_kernel<C, 2><<<grid, 128, 0, s>>>(upper, n, nrhs, A, lda, B, ldb, skip,
                                                          tasks);
        else if(n <= 128)
            cpotrs_warp_kernel<C, 4><<<grid, 128, 0, s>>>(upper, n, nrhs, A, lda, B, ldb, skip,
                                                          tasks);
        else
            cpotrs_warp_kernel<C, 8><<<grid, 128, 0, s>>>(upper, n, nrhs, A, lda, B, ldb, skip,
                                                          tasks);
        return status_of_launch();
    }
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
