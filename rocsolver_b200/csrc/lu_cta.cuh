// lu_cta.cuh -- CTA-per-matrix blocked LU (right-looking, partial pivoting) for
// general m x n.
//
// Replaces the reference's blocked getrf (library/src/lapack/roclapack_getrf.hpp:609-752:
// getrf_panelLU :423-525, getrf_row_permutate :172-210, rocsolver_trsm_lower and the
// rocBLAS GEMM trailing update :721-732), which issues ~100 launches per call at n=256.
//
// B200 design: ONE launch, one CTA per matrix, the whole factorisation in the CTA.
//   * Panel (rows j0..m-1, JB columns) in registers, R rows per thread ("slot").  The
//     column loop is a rolled loop: the active column is always register 0, and the
//     rank-1 update writes element i+1 into register i, so the shift costs nothing and
//     the loop body is one copy of the code (no instruction-cache pressure).  The pivot
//     is a warp redux.sync argmax; each warp publishes its candidate row and the
//     candidate's reciprocal, so ONE __syncthreads per column broadcasts the winner.
//     Row interchanges inside the panel are relabellings; finished L entries (negated)
//     and U rows are parked in shared memory by slot, which is also the A operand of
//     the trailing update.
//   * The panel's interchanges reach the other columns as a warp-local gather/scatter of
//     the moved rows (at most 2*JB) per column, or (fold) only the columns left of it, the
//     trailing update reading each right-hand position from its source row.
//   * U12 = L11^{-1} A12 as a small GEMM: one warp inverts the unit-lower L11 once per
//     panel, then warps multiply 32-column tiles in place in shared memory.
//   * A22 -= L21 U12 as 32x32 warp tiles; A22 is streamed from L2/HBM once per panel.
//   FP64 tiles run on the FP64 tensor path (mma.sync.m8n8k4.f64, 256 FMAs per instruction;
//   tcgen05 has no FP64 kind); FP32 tiles are 4x8 register tiles per lane updated with
//   packed fma.rn.f32x2 (two FMAs per instruction), or, for the mixed solver, split-TF32
//   tensor products (WarpTileTF32).  Shared-memory
//   operands have leading dimension = 4 (mod 16) elements (bank-conflict-free fragments).
#pragma once

#include "common.cuh"
#include "umma.cuh"

namespace rsb {

#ifndef LU_MIN_BLOCKS
#define LU_MIN_BLOCKS 2
#endif
#ifndef LU_MIN_BLOCKS_128
#define LU_MIN_BLOCKS_128 4
#endif
#ifndef LU_CW_F64
#define LU_CW_F64 64
#endif
#ifndef LU_CW_F32
#define LU_CW_F32 128
#endif

template <typename T, int NT, int JB>
struct CtaLuSmem
{
    static constexpr int NW = NT / 32;
    static constexpr int LDI = 36;          // L11 inverse, column-major 32 x 32 (+pad)
    static constexpr int L11LD = 33;        // L11 staging, column-major
    static __host__ __device__ int ldp(int m) { return ((m + 31) / 32) * 32 + 4; }
    static __host__ __device__ int cwp(int cw) { return cw + 4; }
    static __host__ __device__ size_t bytes(int m, int cw, int R)
    {
        using K = typename KeyOf<T>::type;
        size_t s = 0;
        s += sizeof(T) * (size_t)JB * ldp(m);   // panel slots: -L (and U rows), [k][slot]
        s += sizeof(T) * (size_t)JB * cwp(cw);  // A12 / U12 chunk, [k][col]
        s += sizeof(T) * 32 * LDI;              // L11^{-1}
        s += sizeof(T) * 32 * L11LD;            // L11
        s += sizeof(T) * 2 * NW * JB;           // candidate rows
        s += sizeof(T) * 2 * NW;                // candidate reciprocals
        s += sizeof(T) * 2 * NW;                // candidate pivot values
        s += sizeof(K) * 2 * NW;                // candidate keys
        s += sizeof(int) * 2 * NW;              // candidate positions
        s += sizeof(int) * 2 * NW;              // candidate slots
        s += sizeof(int) * (size_t)R * NT;      // slot of each position
        s += sizeof(int) * 4 * JB;              // moved positions and their sources
        s += sizeof(int) * (JB + 2);            // panel pivots, counter
        return (s + 15) & ~size_t(15);
    }
};

// Shared memory of the tcgen05 trailing update (UM variants), placed after CtaLuSmem's
// region (1024-byte aligned): A operand tiles of L21 (groups of um_group() M-tiles of 128
// rows, split TF32 hi and lo), the B operand (a U12 column chunk, hi and lo), an mbarrier and
// the TMEM base address.  One M-tile group's accumulators take um_group() * cw TMEM columns.
template <int NT, int JB>
__host__ __device__ constexpr int um_group_max()
{
    return NT <= 128 ? 1 : (JB >= 32 ? 2 : 4);
}
template <int NT, int JB>
__host__ __device__ inline int um_group(int cw)
{
    const int g = um_group_max<NT, JB>();
    return g * cw <= 512 ? g : (512 / cw > 0 ? 512 / cw : 1);
}
template <int NT, int JB>
__host__ __device__ inline size_t um_bytes(int cw)
{
    return 1024 + sizeof(float) * (size_t)(2 * um_group_max<NT, JB>() * 128 * JB + 2 * cw * JB)
           + 64;
}

// State of the tcgen05 trailing update for one CTA
struct UmCtx
{
    float* ahi;       // [G][128 x JB] K-major split-TF32 tiles of L21
    float* alo;
    float* bhi;       // [cw x JB] K-major split-TF32 U12 chunk
    float* blo;
    uint64_t* mbar;   // MMA completion
    uint32_t tmem;    // TMEM base (G * cw columns)
    int G;
    uint32_t phase;
    int failed;       // an MMA completion wait ran out (CTA-uniform)
};

// ---------------------------------------------------------------------------------------
// Warp tile products.  acc (32 x 32 tile) += A * B over k < K where A(r, k) = sA[k*lda_s +
// arow] (arow: this lane's fragment rows, identity or through the slot table) and
// B(k, c) = sB[k*ldb_s + c0 + c].
template <typename T>
struct WarpTile;

template <>
struct WarpTile<double>
{
    double acc[4][4][2];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for(int mi = 0; mi < 4; ++mi)
#pragma unroll
            for(int ni = 0; ni < 4; ++ni)
                acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
    }
    template <int K>
    __device__ __forceinline__ void mma(const double* sA, int lda_s, const int (&arow)[4],
                                        const double* sB, int ldb_s, int c0)
    {
        const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
#pragma unroll 2
        for(int k0 = 0; k0 < K; k0 += 4)
        {
            double af[4], bf[4];
#pragma unroll
            for(int mi = 0; mi < 4; ++mi)
                af[mi] = sA[(k0 + tq) * lda_s + arow[mi]];
#pragma unroll
            for(int ni = 0; ni < 4; ++ni)
                bf[ni] = sB[(k0 + tq) * ldb_s + c0 + ni * 8 + g];
#pragma unroll
            for(int mi = 0; mi < 4; ++mi)
#pragma unroll
                for(int ni = 0; ni < 4; ++ni)
                    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
                                 "{%0, %1}, {%2}, {%3}, {%0, %1};\n"
                                 : "+d"(acc[mi][ni][0]), "+d"(acc[mi][ni][1])
                                 : "d"(af[mi]), "d"(bf[ni]));
        }
    }
    // visit every tile element this lane holds: f(row in tile, col in tile, value&)
    template <typename F>
    __device__ __forceinline__ void each(F f)
    {
        const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
#pragma unroll
        for(int mi = 0; mi < 4; ++mi)
#pragma unroll
            for(int ni = 0; ni < 4; ++ni)
#pragma unroll
                for(int e = 0; e < 2; ++e)
                    f(mi * 8 + g, ni * 8 + tq * 2 + e, acc[mi][ni][e]);
    }
    static __device__ __forceinline__ int frag_row(int mi)
    {
        return mi * 8 + ((threadIdx.x & 31) >> 2);
    }
};

// acc(i, 2p..2p+1) += l(i) * (u(2p), u(2p+1)) as one packed FP32 FMA (fma.rn.f32x2: each
// half rounds exactly like fmaf, so results equal the scalar form bit for bit)
__device__ __forceinline__ void fma2(float2& acc, float l, float u0, float u1)
{
    asm("{\n\t.reg .b64 pa, pb, pc;\n\t"
        "mov.b64 pa, {%2, %2};\n\t"
        "mov.b64 pb, {%3, %4};\n\t"
        "mov.b64 pc, {%0, %1};\n\t"
        "fma.rn.f32x2 pc, pa, pb, pc;\n\t"
        "mov.b64 {%0, %1}, pc;\n\t}"
        : "+f"(acc.x), "+f"(acc.y)
        : "f"(l), "f"(u0), "f"(u1));
}

template <>
struct WarpTile<float>
{
    float2 acc[4][4]; // rows rg*4+i, columns cg*8 + 2p + {0,1}
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for(int i = 0; i < 4; ++i)
#pragma unroll
            for(int p = 0; p < 4; ++p)
                acc[i][p] = make_float2(0.f, 0.f);
    }
    template <int K>
    __device__ __forceinline__ void mma(const float* sA, int lda_s, const int (&arow)[4],
                                        const float* sB, int ldb_s, int c0)
    {
        const int cg = (threadIdx.x & 31) >> 3;
#pragma unroll 4
        for(int k = 0; k < K; ++k)
        {
            float lv[4];
#pragma unroll
            for(int i = 0; i < 4; ++i)
                lv[i] = sA[k * lda_s + arow[i]];
            const float4 u0 = *reinterpret_cast<const float4*>(sB + k * ldb_s + c0 + cg * 8);
            const float4 u1 = *reinterpret_cast<const float4*>(sB + k * ldb_s + c0 + cg * 8 + 4);
#pragma unroll
            for(int i = 0; i < 4; ++i)
            {
                fma2(acc[i][0], lv[i], u0.x, u0.y);
                fma2(acc[i][1], lv[i], u0.z, u0.w);
                fma2(acc[i][2], lv[i], u1.x, u1.y);
                fma2(acc[i][3], lv[i], u1.z, u1.w);
            }
        }
    }
    template <typename F>
    __device__ __forceinline__ void each(F f)
    {
        const int lane = threadIdx.x & 31, rg = lane & 7, cg = lane >> 3;
#pragma unroll
        for(int i = 0; i < 4; ++i)
#pragma unroll
            for(int p = 0; p < 4; ++p)
            {
                f(rg * 4 + i, cg * 8 + 2 * p, acc[i][p].x);
                f(rg * 4 + i, cg * 8 + 2 * p + 1, acc[i][p].y);
            }
    }
    static __device__ __forceinline__ int frag_row(int i)
    {
        return ((threadIdx.x & 31) & 7) * 4 + i;
    }
};

// Round to TF32 (nearest, ties away from zero): half a TF32 unit added to the magnitude
// bits, the 13 low mantissa bits cleared.  Integer operations only (the conversion
// instruction runs on the narrow transcendental pipe).  Finite inputs near the FP32 limit
// round to infinity, as the conversion does.
__device__ __forceinline__ uint32_t tf32_rna(float x)
{
    return (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
}

// x = hi + lo + O(2^-24 |x|): hi = x rounded to TF32, lo = (x - hi) (exact in FP32) rounded
// to TF32
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo)
{
    hi = tf32_rna(x);
    lo = tf32_rna(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1)
{
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 "
        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// FP32 tile product on the TF32 tensor path at FP32-level accuracy (split TF32, three
// products): a = a_hi + a_lo, b = b_hi + b_lo, a*b ~ a_lo*b_hi + a_hi*b_lo + a_hi*b_hi
// accumulated in FP32 (the dropped a_lo*b_lo is below 2^-21 |a||b|).  A 32 x 32 warp tile
// is 2 x 4 blocks of mma.sync.m16n8k8 .tf32 (lane = 4*g + q holds rows g, g+8 of each
// 16-row block and columns 2q, 2q+1 of each 8-column block); per 8-deep k step a lane
// loads 16 operands (bank-conflict-free with leading dimensions = 4 mod 32) for 24 tensor
// instructions, against 128 packed FMAs for the same step on CUDA cores.  Used for the
// trailing update of the mixed solver's FP32 factorisation, where accuracy only sets the
// refinement's convergence rate.
struct WarpTileTF32
{
    float acc[2][4][4]; // [16-row block][8-column block][fragment element]
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for(int mi = 0; mi < 2; ++mi)
#pragma unroll
            for(int ni = 0; ni < 4; ++ni)
#pragma unroll
                for(int e = 0; e < 4; ++e)
                    acc[mi][ni][e] = 0.f;
    }
    // arow[2*mi + h]: shared-memory row of tile row 16*mi + 8*h + g (see frag_row)
    template <int K>
    __device__ __forceinline__ void mma(const float* sA, int lda_s, const int (&arow)[4],
                                        const float* sB, int ldb_s, int c0)
    {
        static_assert(K % 8 == 0, "TF32 k step is 8");
        const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll 1
        for(int k0 = 0; k0 < K; k0 += 8)
        {
            uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
            // A fragment element e: row g + 8*(e&1), k q + 4*(e>>1)
#pragma unroll
            for(int mi = 0; mi < 2; ++mi)
#pragma unroll
                for(int e = 0; e < 4; ++e)
                    tf32_split(sA[(k0 + q + 4 * (e >> 1)) * lda_s + arow[mi * 2 + (e & 1)]],
                               ah[mi][e], al[mi][e]);
            // B fragment element e: k q + 4*e, column g
#pragma unroll
            for(int ni = 0; ni < 4; ++ni)
#pragma unroll
                for(int e = 0; e < 2; ++e)
                    tf32_split(sB[(k0 + q + 4 * e) * ldb_s + c0 + ni * 8 + g], bh[ni][e],
                               bl[ni][e]);
            // small products first; eight independent blocks between dependent products
#pragma unroll
            for(int mi = 0; mi < 2; ++mi)
#pragma unroll
                for(int ni = 0; ni < 4; ++ni)
                    mma_tf32(acc[mi][ni], al[mi], bh[ni][0], bh[ni][1]);
#pragma unroll
            for(int mi = 0; mi < 2; ++mi)
#pragma unroll
                for(int ni = 0; ni < 4; ++ni)
                    mma_tf32(acc[mi][ni], ah[mi], bl[ni][0], bl[ni][1]);
#pragma unroll
            for(int mi = 0; mi < 2; ++mi)
#pragma unroll
                for(int ni = 0; ni < 4; ++ni)
                    mma_tf32(acc[mi][ni], ah[mi], bh[ni][0], bh[ni][1]);
        }
    }
    // accumulator element e of block (mi, ni): row 16*mi + g + 8*(e>>1), column
    // 8*ni + 2*q + (e&1)
    template <typename F>
    __device__ __forceinline__ void each(F f)
    {
        const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll
        for(int mi = 0; mi < 2; ++mi)
#pragma unroll
            for(int ni = 0; ni < 4; ++ni)
#pragma unroll
                for(int e = 0; e < 4; ++e)
                    f(mi * 16 + g + 8 * (e >> 1), ni * 8 + 2 * q + (e & 1), acc[mi][ni][e]);
    }
    static __device__ __forceinline__ int frag_row(int i)
    {
        return (i >> 1) * 16 + (i & 1) * 8 + ((threadIdx.x & 31) >> 2);
    }
};

// tile type of the trailing update: TC selects the split-TF32 tensor path for FP32
// (panel widths that are multiples of the 8-deep TF32 k step)
template <typename T, bool TC>
struct TileOf
{
    using type = WarpTile<T>;
};
template <>
struct TileOf<float, true>
{
    using type = WarpTileTF32;
};

// A22 += L21 U12 on tcgen05 for one panel (rows already interchanged in memory, U12 stored in
// the panel's top rows j0..j0+jb-1).  A22 = rows j0+jb.. (mt of them), columns j0+jb..n-1.
// sP holds -L by slot ([k][slot], leading dimension ldp); A22 row r takes L21 row slotof[jb+r].
// M-tiles of 128 rows are processed G at a time: their split-TF32 L21 tiles are built once,
// then for each column chunk of at most cw columns the U12 chunk is split into the B operand,
// one thread issues 3 * (JB/8) MMAs per M-tile into TMEM (columns t*cw.. of tile t), commits
// to the mbarrier, and after the (bounded) wait every warp adds its TMEM rows into A22 with
// coalesced column accesses (warp w reads TMEM lanes 32*(w%4)..+31 of the tiles of its
// warpgroup).  All threads of the CTA call it.
template <int NT, int JB>
__device__ __noinline__ void umma_update(float* a, int lda, int j0, int jb, int mt, int n,
                                         const float* sP, int ldp, const int* slotof, int cw,
                                         UmCtx& um)
{
    const int c_first = j0 + jb;
    if(mt <= 0 || c_first >= n || um.failed)
        return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int TILE = 128 * JB;          // floats per M-tile operand
    constexpr uint32_t SBO = (JB / 4) * 128; // bytes between 8-row groups
    const int mtiles = (mt + 127) / 128;
    const int G = um.G;
    const uint32_t ahi = umma::smem_u32(um.ahi), alo = umma::smem_u32(um.alo);
    const uint32_t bhi = umma::smem_u32(um.bhi), blo = umma::smem_u32(um.blo);
    for(int g0 = 0; g0 < mtiles && !um.failed; g0 += G)
    {
        const int gt = min(G, mtiles - g0);
        // L21 tiles of this group: row r (A22 position jb + r) from slot slotof[jb + r]
        for(int e = tid; e < gt * 128 * JB; e += NT)
        {
            const int rr = e % (gt * 128), k = e / (gt * 128);
            const int t = rr >> 7, rl = rr & 127, r = g0 * 128 + rr;
            const float x = (r < mt && k < jb) ? sP[k * ldp + slotof[jb + r]] : 0.f;
            uint32_t h, l;
            umma::split_tf32(x, h, l);
            const uint32_t off = umma::kmaj_off(rl, k, JB) >> 2;
            reinterpret_cast<uint32_t*>(um.ahi + t * TILE)[off] = h;
            reinterpret_cast<uint32_t*>(um.alo + t * TILE)[off] = l;
        }
        for(int c0 = c_first; c0 < n && !um.failed; c0 += cw)
        {
            const int ncol = min(cw, n - c0);
            const int ncp = (ncol + 31) & ~31;
            // U12 chunk (the panel's top rows, just stored) -> B operand
            for(int e = tid; e < ncp * JB; e += NT)
            {
                const int k = e % JB, col = e / JB;
                const float x = (k < jb && col < ncol) ? a[ix(j0 + k, c0 + col, lda)] : 0.f;
                uint32_t h, l;
                umma::split_tf32(x, h, l);
                const uint32_t off = umma::kmaj_off(col, k, JB) >> 2;
                reinterpret_cast<uint32_t*>(um.bhi)[off] = h;
                reinterpret_cast<uint32_t*>(um.blo)[off] = l;
            }
            umma::fence_async_shared();
            umma::fence_before_sync();
            __syncthreads();
            umma::fence_after_sync();
            if(tid == 0)
            {
                const uint32_t idesc = umma::idesc_tf32(128, ncp);
                for(int t = 0; t < gt; ++t)
                {
                    const uint32_t d = um.tmem + (uint32_t)(t * cw);
#pragma unroll
                    for(int s = 0; s < JB / 8; ++s)
                    {
                        const uint32_t ao = (uint32_t)(t * TILE * 4 + 256 * s), bo = 256u * s;
                        umma::mma_tf32(d, umma::sdesc(alo + ao, 128, SBO),
                                       umma::sdesc(bhi + bo, 128, SBO), idesc, s > 0 ? 1u : 0u);
                        umma::mma_tf32(d, umma::sdesc(ahi + ao, 128, SBO),
                                       umma::sdesc(blo + bo, 128, SBO), idesc, 1u);
                        umma::mma_tf32(d, umma::sdesc(ahi + ao, 128, SBO),
                                       umma::sdesc(bhi + bo, 128, SBO), idesc, 1u);
                    }
                }
                umma::commit(um.mbar);
            }
            const bool ok = umma::mbar_wait(um.mbar, um.phase);
            um.phase ^= 1u;
            if(__syncthreads_or(ok ? 0 : 1))
            {
                um.failed = 1;
                break;
            }
            umma::fence_after_sync();
            // epilogue: A22 rows of this warp's TMEM lanes += their accumulators
            for(int t = warp >> 2; t < gt; t += NT / 128)
            {
                const int row = (g0 + t) * 128 + (warp & 3) * 32 + lane;
                for(int cb = 0; cb < ncp; cb += 16)
                {
                    float v[16];
                    umma::tmem_ld16(um.tmem + ((uint32_t)((warp & 3) * 32) << 16)
                                        + (uint32_t)(t * cw + cb),
                                    v);
                    if(row < mt)
                    {
                        float* dst = a + ix(j0 + jb + row, c0 + cb, lda);
                        float old[16];
#pragma unroll
                        for(int j = 0; j < 16; ++j)
                            old[j] = cb + j < ncol ? dst[(size_t)j * lda] : 0.f;
#pragma unroll
                        for(int j = 0; j < 16; ++j)
                            if(cb + j < ncol)
                                dst[(size_t)j * lda] = old[j] + v[j];
                    }
                }
            }
            umma::fence_before_sync();
            __syncthreads(); // the B operand and TMEM are reused by the next chunk
        }
    }
}

// Factor one m x n matrix with the whole CTA.  smem_raw must hold CtaLuSmem::bytes(m, cw, R);
// m <= R*NT; cw is a multiple of 32.  Writes ipiv (1-based, PIVOT only) and *info_out.
// fold: apply each panel's row interchanges to the columns right of it inside the trailing
// update instead of swapping them in memory first (a tuning choice; same results).
// TC: FP32 trailing products on the split-TF32 tensor path (WarpTileTF32).
// Called by all threads of the CTA.
// UM (FP32 with TC and PIVOT, JB a multiple of 8): the trailing update A22 += L21 U12 runs
// on tcgen05 (umma_update below) with the rows interchanged in memory first (no fold) and
// U12 stored before it; um holds its buffers and TMEM.
template <typename T, int NT, int R, int JB, int TN, bool PIVOT, bool TC = false,
          bool UM = false>
__device__ __forceinline__ void getrf_cta_dev(int m, int n, T* a, int lda, int* piv_out,
                                              int* info_out, int cw, bool fold_arg,
                                              unsigned char* smem_raw, UmCtx* um = nullptr)
{
    static_assert(!UM || (sizeof(T) == 4 && TC && PIVOT && JB % 8 == 0), "tcgen05 variant");
    const bool fold = UM ? false : fold_arg;
    static_assert(JB % 4 == 0 && JB <= 32, "panel width");
    static_assert(NT % 32 == 0 && NT <= 1024, "CTA size");
    using K = typename KeyOf<T>::type;
    using SM = CtaLuSmem<T, NT, JB>;
    using Tile = typename TileOf<T, TC && JB % 8 == 0>::type;
    constexpr int NW = NT / 32;
    const int ldp = SM::ldp(m), cwp = SM::cwp(cw);
    T* sP = reinterpret_cast<T*>(smem_raw);          // [JB][ldp]
    T* sU = sP + (size_t)JB * ldp;                     // [JB][cwp]
    T* sLi = sU + (size_t)JB * cwp;                    // [32][LDI]
    T* sL11 = sLi + 32 * SM::LDI;                      // [32][L11LD]
    T* cand = sL11 + 32 * SM::L11LD;                   // [2][NW][JB]
    T* crcp = cand + 2 * NW * JB;                      // [2][NW]
    T* cpiv = crcp + 2 * NW;                           // [2][NW]
    K* ckey = reinterpret_cast<K*>(cpiv + 2 * NW);     // [2][NW]
    int* crow = reinterpret_cast<int*>(ckey + 2 * NW); // [2][NW]
    int* cslot = crow + 2 * NW;                        // [2][NW]
    int* slotof = cslot + 2 * NW;                      // [R*NT]
    int* moved = slotof + R * NT;                      // [2*JB]
    int* movsrc = moved + 2 * JB;                      // [2*JB]
    int* spiv = movsrc + 2 * JB;                       // [JB]
    int* nmoved = spiv + JB;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mn = min(m, n);
    int inf = 0;

    for(int j0 = 0; j0 < mn; j0 += JB)
    {
        const int jb = min(JB, mn - j0);
        const int mp = m - j0;
        T pv[R][JB];
        int lrow[R];
        // ---------------- load the panel (rows j0..m-1, columns j0..j0+jb-1)
#pragma unroll
        for(int q = 0; q < R; ++q)
        {
            const int r = tid + q * NT;
            lrow[q] = r;
#pragma unroll
            for(int c = 0; c < JB; ++c)
                pv[q][c] = (r < mp && c < jb) ? RSB_AT(a, j0 + r, j0 + c, lda, m, n) : T(0);
        }
        // ---------------- factor the panel: rolled column loop, one barrier per column.
        // Warps whose slots all lie below the panel's last row only keep the barrier.
        const int nact = min(NW, (mp + 31) / 32);
        if(warp >= nact)
        {
#pragma unroll 1
            for(int c = 0; c < jb; ++c)
                __syncthreads();
        }
        else
#pragma unroll 1
        for(int c = 0; c < jb; ++c)
        {
            const int buf = c & 1;
            T* cb = cand + buf * NW * JB;
            int prow = c, gw = 0;
            if(PIVOT)
            {
                K bk = 0;
                int br = INT_MAX;
                T bv = T(0);
                bool any = false;
#pragma unroll
                for(int q = 0; q < R; ++q)
                {
                    if(tid + q * NT < mp && lrow[q] >= c)
                    {
                        const K kq = pivot_key(pv[q][0], lrow[q] == c);
                        if(!any || kq > bk || (kq == bk && lrow[q] < br))
                        {
                            bk = kq;
                            br = lrow[q];
                            bv = pv[q][0];
                            any = true;
                        }
                    }
                }
                // the candidate's reciprocal, formed while the reductions run (off the
                // column's serial path)
                const T brc = bv != T(0) ? Lim<T>::rcp(bv) : T(0);
                K wk;
                const int wr = warp_argmax(bk, br, any, &wk);
                if(any && br == wr)
                {
#pragma unroll
                    for(int q = 0; q < R; ++q)
                        if(lrow[q] == wr && tid + q * NT < mp)
                        {
                            store_row_shifted<T, JB>(cb + warp * JB, pv[q]);
                            cpiv[buf * NW + warp] = pv[q][0];
                            crcp[buf * NW + warp] = brc;
                            cslot[buf * NW + warp] = tid + q * NT;
                        }
                }
                if(lane == 0)
                {
                    ckey[buf * NW + warp] = wk;
                    crow[buf * NW + warp] = wr;
                }
                __syncthreads();
                // the warps' records are reduced lane-parallel (lane w holds warp w's
                // record): largest key, smallest position on ties (LAPACK: first index of
                // the maximum); gw = the warp that published the winning row
                const bool rv = lane < nact;
                const K kl = rv ? ckey[buf * NW + lane] : K(0);
                const int rl = rv ? crow[buf * NW + lane] : INT_MAX;
                K gk;
                const int gr = warp_argmax(kl, rl, rv && rl != INT_MAX, &gk);
                gw = __ffs(__ballot_sync(0xffffffffu, rv && rl == gr && kl == gk)) - 1;
                if(gw < 0)
                    gw = 0;
                prow = gr;
            }
            else
            {
#pragma unroll
                for(int q = 0; q < R; ++q)
                    if(lrow[q] == c && tid + q * NT < mp)
                    {
                        store_row_shifted<T, JB>(cb, pv[q]);
                        const T p = pv[q][0];
                        cpiv[buf * NW] = p;
                        crcp[buf * NW] = p != T(0) ? Lim<T>::rcp(p) : T(0);
                    }
                __syncthreads();
            }
            const T* prowv = cb + gw * JB; // pivot row, shifted by one
            const T pivv = cpiv[buf * NW + gw];
            const T rcp = crcp[buf * NW + gw];
            // row c of U: the pivot row's remaining panel entries, one per lane of the
            // publishing warp (prowv holds columns c+1.. of the pivot row)
            if(warp == gw && lane < jb - c)
                sP[(c + lane) * ldp + (PIVOT ? cslot[buf * NW + gw] : c)] =
                    lane == 0 ? pivv : prowv[lane - 1];
            if(tid == 0)
                spiv[c] = prow;
            if(pivv == T(0) && inf == 0)
                inf = j0 + c + 1;
            // LAPACK getf2 scaling: reciprocal when |pivot| >= sfmin, else division
            const int mode = pivv == T(0) ? 0 : (fabs(pivv) >= Lim<T>::sfmin() ? 1 : 2);
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
                const int slot = tid + q * NT;
                if(slot < mp)
                {
                    if(lrow[q] > c)
                    {
                        const T x = pv[q][0];
                        const T l = mode == 1 ? x * rcp : (mode == 2 ? x / pivv : x);
                        sP[c * ldp + slot] = -l;
                        update_shift<T, JB>(pv[q], l, prowv, jb - c - 2);
                    }
                }
            }
        }
        __syncthreads();
        // ---------------- panel write-back at final positions; slot table; L11
#pragma unroll
        for(int q = 0; q < R; ++q)
        {
            const int slot = tid + q * NT;
            if(slot < mp)
            {
                const int pos = lrow[q];
#pragma unroll 4
                for(int k = 0; k < jb; ++k)
                {
                    const T v = sP[k * ldp + slot];
                    RSB_AT(a, j0 + pos, j0 + k, lda, m, n) = k < pos ? -v : v;
                }
                slotof[pos] = slot;
            }
        }
        if(tid == 0)
            *nmoved = 0;
        __syncthreads();
        for(int e = tid; e < 32 * 32; e += NT)
        {
            const int i = e & 31, k = e >> 5; // L11(i, k), unit lower
            T v = T(0);
            if(i < jb && k < jb)
                v = i > k ? -sP[k * ldp + slotof[i]] : (i == k ? T(1) : T(0));
            sL11[k * SM::L11LD + i] = v;
        }
        if(PIVOT)
        {
            if(tid < jb)
                piv_out[j0 + tid] = j0 + spiv[tid] + 1;
            for(int p = tid; p < mp; p += NT)
            {
                const int s = slotof[p];
                if(s != p)
                {
                    const int idx = atomicAdd(nmoved, 1);
                    moved[idx] = p;
                    movsrc[idx] = s;
                }
            }
        }
        __syncthreads();
        // ---------------- L11^{-1}: lane j solves L11 x = e_j (column j of the inverse)
        if(warp == 0)
        {
            T x[32];
#pragma unroll
            for(int i = 0; i < 32; ++i)
                x[i] = (i == lane && lane < jb) ? T(1) : T(0);
#pragma unroll
            for(int k = 0; k < 32; ++k)
#pragma unroll
                for(int i = k + 1; i < 32; ++i)
                    x[i] = fma(-sL11[k * SM::L11LD + i], x[k], x[i]);
#pragma unroll
            for(int i = 0; i < 32; ++i)
                sLi[lane * SM::LDI + i] = x[i];
        }
        // ---------------- row interchanges: warp-local gather/scatter of the moved rows, 4
        // columns per batch, on the columns left of the panel (finished L) and, unless they
        // are folded into the trailing update, on the columns right of it
        const int nm = PIVOT ? *nmoved : 0;
        const int nother = fold ? j0 : n - jb;
        if(nm > 0)
        {
            for(int o0 = warp * 4; o0 < nother; o0 += NW * 4)
            {
                T v[4][2];
#pragma unroll
                for(int u = 0; u < 4; ++u)
                {
                    const int o = o0 + u;
                    const int col = o < j0 ? o : o + jb;
#pragma unroll
                    for(int s = 0; s < 2; ++s)
                    {
                        const int i = lane + 32 * s;
                        if(o < nother && i < nm)
                            v[u][s] = RSB_AT(a, j0 + movsrc[i], col, lda, m, n);
                    }
                }
                __syncwarp();
#pragma unroll
                for(int u = 0; u < 4; ++u)
                {
                    const int o = o0 + u;
                    const int col = o < j0 ? o : o + jb;
#pragma unroll
                    for(int s = 0; s < 2; ++s)
                    {
                        const int i = lane + 32 * s;
                        if(o < nother && i < nm)
                            RSB_AT(a, j0 + moved[i], col, lda, m, n) = v[u][s];
                    }
                }
            }
        }
        __syncthreads();
        // ---------------- trailing update, column chunk by column chunk.  With fold, the
        // panel's row interchanges are applied here: position p of the chunk receives the
        // original row slotof[p].  A position below the panel rows (p >= jb) either keeps
        // its row or receives an original top row (p < jb): a row only moves down when it
        // sits in the position of the column being pivoted, and only top positions are
        // pivoted.  So:
        //   1. stage A12 from the sources of the top positions (reads only, into sU);
        //   2. U12 = L11^{-1} A12 in sU;
        //   3. A22 tiles read position p from global row slotof[p] (itself or an untouched
        //      top row) and write position p: no position is read after it is written;
        //   4. U12 goes to the top rows last, once no tile needs their original values.
        // Without fold the rows are already in place and U12 is stored as it is formed.
        const int mt = mp - jb;
        for(int c0 = j0 + jb; c0 < n; c0 += cw)
        {
            const int ncol = min(cw, n - c0);
            const int ncp = (ncol + 31) & ~31;
            // loads of 4 elements issued before their stores (overlapped latency)
            for(int e0 = tid; e0 < JB * ncp; e0 += 4 * NT)
            {
                T t[4];
#pragma unroll
                for(int u = 0; u < 4; ++u)
                {
                    const int e = e0 + u * NT, k = e % JB, col = e / JB;
                    t[u] = (e < JB * ncp && k < jb && col < ncol)
                               ? RSB_AT(a, j0 + (fold ? slotof[k] : k), c0 + col, lda, m, n)
                               : T(0);
                }
#pragma unroll
                for(int u = 0; u < 4; ++u)
                {
                    const int e = e0 + u * NT;
                    if(e < JB * ncp)
                        sU[(e % JB) * cwp + e / JB] = t[u];
                }
            }
            __syncthreads();
            for(int t = warp; t < ncp / 32; t += NW)
            {
                Tile w;
                w.zero();
                int arow[4];
#pragma unroll
                for(int mi = 0; mi < 4; ++mi)
                    arow[mi] = Tile::frag_row(mi);
                w.template mma<JB>(sLi, SM::LDI, arow, sU, cwp, t * 32);
                __syncwarp();
                w.each([&](int rr, int cc, T& v) {
                    const int col = t * 32 + cc;
                    if(rr < JB)
                        sU[rr * cwp + col] = rr < jb ? v : T(0);
                    if(!fold && rr < jb && col < ncol)
                        RSB_AT(a, j0 + rr, c0 + col, lda, m, n) = v;
                });
            }
            __syncthreads();
            // A22 -= L21 U12: 32x32 tiles of (mt x ncol); L21 rows through the slot table
            // (the UM variant updates A22 after the chunk loop, on tcgen05)
            const int tm = UM ? 0 : (mt + 31) / 32, tn = ncp / 32;
            for(int t = warp; t < tm * tn; t += NW)
            {
                const int tmd = tm > 0 ? tm : 1; // tm == 0 (UM) never enters the loop
                const int r0 = (t % tmd) * 32, cc0 = (t / tmd) * 32;
                Tile w;
                int arow[4];
#pragma unroll
                for(int mi = 0; mi < 4; ++mi)
                {
                    const int r = r0 + Tile::frag_row(mi);
                    arow[mi] = r < mt ? slotof[jb + r] : 0;
                }
                w.each([&](int rr, int cc, T& v) {
                    const int r = r0 + rr, col = cc0 + cc;
                    v = (r < mt && col < ncol)
                            ? RSB_AT(a, j0 + (fold ? slotof[jb + r] : jb + r), c0 + col, lda, m, n)
                            : T(0);
                });
                w.template mma<JB>(sP, ldp, arow, sU, cwp, cc0);
                w.each([&](int rr, int cc, T& v) {
                    const int r = r0 + rr, col = cc0 + cc;
                    if(r < mt && col < ncol)
                        RSB_AT(a, j0 + jb + r, c0 + col, lda, m, n) = v;
                });
            }
            __syncthreads();
            if(fold)
            {
                for(int e = tid; e < JB * ncol; e += NT)
                {
                    const int k = e % JB, col = e / JB;
                    if(k < jb)
                        RSB_AT(a, j0 + k, c0 + col, lda, m, n) = sU[k * cwp + col];
                }
                __syncthreads();
            }
        }
        if constexpr(UM)
            umma_update<NT, JB>(a, lda, j0, jb, mt, n, reinterpret_cast<const float*>(sP), ldp,
                                slotof, cw, *um);
    }
    if constexpr(UM)
        if(um->failed && tid == 0)
            inf = INT_MIN; // a tensor-core completion wait ran out: results are not valid
    if(tid == 0)
        *info_out = inf;
}

// ---------------------------------------------------------------------------------------
// Two-level blocking for large orders (FP32, split TF32 on tcgen05).  Outer panels of JO = 64
// columns are factored by getrf_cta_dev itself (register panels of JB columns whose trailing
// updates stay inside the outer panel, which is L2-resident), then the outer panel's row
// interchanges reach the other columns, U12 = L11^{-1} A12 is formed by forward
// substitution, and A22 -= L21 U12 runs once per outer panel with K = 64 on tcgen05
// (umma_update_k64): A22 is streamed once per 64 columns instead of once per JB.

constexpr int LU2_JO = 64; // outer panel width (the K of the tcgen05 trailing update)

// Shared memory of the two-level variant after CtaLuSmem's region: one 128-row M-tile of
// L21 (hi and lo, K = 64), the U12 chunk (hi and lo), mbarrier.  The forward substitution
// stages L11 (64 x 65 floats) in the M-tile's space.
__host__ __device__ inline size_t lu2_bytes(int cw)
{
    return 1024 + sizeof(float) * (size_t)(2 * 128 * LU2_JO + 2 * cw * LU2_JO) + 64;
}

// A22 += L21 U12 with K = kk <= 64 on tcgen05, all operands in global memory (column-major,
// leading dimension lda): A22 = a[r0 + r, c] for r < mt and cfirst <= c < n, L21(r, k) =
// a[r0 + r, kc0 + k], U12(k, c) = a[kr0 + k, c].  Same structure as umma_update with one
// M-tile per MMA group (um.G = 1).  All threads of the CTA call it.
template <int NT>
__device__ __noinline__ void umma_update_k64(float* a, int lda, int r0, int kc0, int kr0,
                                             int kk, int mt, int cfirst, int n, int cw,
                                             UmCtx& um)
{
    constexpr int KK = LU2_JO;
    constexpr uint32_t SBO = (KK / 4) * 128;
    if(mt <= 0 || cfirst >= n || um.failed)
        return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ahi = umma::smem_u32(um.ahi), alo = umma::smem_u32(um.alo);
    const uint32_t bhi = umma::smem_u32(um.bhi), blo = umma::smem_u32(um.blo);
    const int mtiles = (mt + 127) / 128;
    for(int t = 0; t < mtiles && !um.failed; ++t)
    {
        // this M-tile's L21 rows, negated (A22 -= L21 U12 is accumulated as A22 + (-L21) U12;
        // rows fastest: coalesced column reads)
        for(int e = tid; e < 128 * KK; e += NT)
        {
            const int rl = e & 127, k = e >> 7, r = t * 128 + rl;
            const float x = (r < mt && k < kk) ? -a[ix(r0 + r, kc0 + k, lda)] : 0.f;
            uint32_t h, l;
            umma::split_tf32(x, h, l);
            const uint32_t off = umma::kmaj_off(rl, k, KK) >> 2;
            reinterpret_cast<uint32_t*>(um.ahi)[off] = h;
            reinterpret_cast<uint32_t*>(um.alo)[off] = l;
        }
        for(int c0 = cfirst; c0 < n && !um.failed; c0 += cw)
        {
            const int ncol = min(cw, n - c0);
            const int ncp = (ncol + 31) & ~31;
            for(int e = tid; e < ncp * KK; e += NT)
            {
                const int k = e % KK, col = e / KK;
                const float x = (k < kk && col < ncol) ? a[ix(kr0 + k, c0 + col, lda)] : 0.f;
                uint32_t h, l;
                umma::split_tf32(x, h, l);
                const uint32_t off = umma::kmaj_off(col, k, KK) >> 2;
                reinterpret_cast<uint32_t*>(um.bhi)[off] = h;
                reinterpret_cast<uint32_t*>(um.blo)[off] = l;
            }
            umma::fence_async_shared();
            umma::fence_before_sync();
            __syncthreads();
            umma::fence_after_sync();
            if(tid == 0)
            {
                const uint32_t idesc = umma::idesc_tf32(128, ncp);
#pragma unroll
                for(int s = 0; s < KK / 8; ++s)
                {
                    const uint32_t o = 256u * s;
                    umma::mma_tf32(um.tmem, umma::sdesc(alo + o, 128, SBO),
                                   umma::sdesc(bhi + o, 128, SBO), idesc, s > 0 ? 1u : 0u);
                    umma::mma_tf32(um.tmem, umma::sdesc(ahi + o, 128, SBO),
                                   umma::sdesc(blo + o, 128, SBO), idesc, 1u);
                    umma::mma_tf32(um.tmem, umma::sdesc(ahi + o, 128, SBO),
                                   umma::sdesc(bhi + o, 128, SBO), idesc, 1u);
                }
                umma::commit(um.mbar);
            }
            // epilogue: thread (warp w, lane) owns A22 row t*128 + 32*(w%4) + lane (its TMEM
            // lane); warpgroup g takes the 16-column blocks g, g + NWG, ...  The first block's
            // A22 values are loaded while the MMAs run, each next block's before the current
            // one is stored.
            constexpr int NWG = NT / 128;
            const int wg = warp >> 2;
            const int row = t * 128 + (warp & 3) * 32 + lane;
            const bool mine = row < mt;
            float* dst = a + ix(r0 + (mine ? row : 0), c0, lda);
            float pre[16];
#pragma unroll
            for(int j = 0; j < 16; ++j)
                pre[j] = (mine && wg * 16 + j < ncol) ? dst[(size_t)(wg * 16 + j) * lda] : 0.f;
            const bool ok = umma::mbar_wait(um.mbar, um.phase);
            um.phase ^= 1u;
            if(__syncthreads_or(ok ? 0 : 1))
            {
                um.failed = 1;
                break;
            }
            umma::fence_after_sync();
            for(int cb = wg * 16; cb < ncp; cb += 16 * NWG)
            {
                float v[16];
                umma::tmem_ld16(um.tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)cb, v);
                const int cn = cb + 16 * NWG;
                float nxt[16];
#pragma unroll
                for(int j = 0; j < 16; ++j)
                    nxt[j] = (mine && cn + j < ncol) ? dst[(size_t)(cn + j) * lda] : 0.f;
                if(mine)
                {
#pragma unroll
                    for(int j = 0; j < 16; ++j)
                        if(cb + j < ncol)
                            dst[(size_t)(cb + j) * lda] = pre[j] + v[j];
                }
#pragma unroll
                for(int j = 0; j < 16; ++j)
                    pre[j] = nxt[j];
            }
            umma::fence_before_sync();
            __syncthreads();
        }
    }
}

// U12 = L11^{-1} A12 in place for the outer panel at (j0, j0) of width jo <= 64 (L11 unit
// lower, staged in shared memory sl as [i][k] with leading dimension 65): one thread per
// column, in two halves of 32 rows (top: x = L00^{-1} a_top; bottom: a_bot -= L10 x, then
// x' = L11^{-1} a_bot), the column held in registers.
template <int NT>
__device__ __noinline__ void lu2_trsm(float* a, int lda, int j0, int jo, int n, float* sl)
{
    constexpr int LD = LU2_JO + 1;
    for(int e = threadIdx.x; e < LU2_JO * LU2_JO; e += NT)
    {
        const int i = e % LU2_JO, k = e / LU2_JO;
        sl[i * LD + k] = (i < jo && i > k) ? a[ix(j0 + i, j0 + k, lda)] : 0.f;
    }
    __syncthreads();
    for(int c = j0 + jo + threadIdx.x; c < n; c += NT)
    {
        float* col = a + ix(j0, c, lda);
        float x[32];
#pragma unroll
        for(int i = 0; i < 32; ++i)
            x[i] = i < jo ? col[i] : 0.f;
#pragma unroll
        for(int k = 0; k < 32; ++k)
#pragma unroll
            for(int i = k + 1; i < 32; ++i)
                x[i] = fmaf(-sl[i * LD + k], x[k], x[i]);
#pragma unroll
        for(int i = 0; i < 32; ++i)
            if(i < jo)
                col[i] = x[i];
        if(jo > 32)
        {
            float y[32];
#pragma unroll
            for(int i = 0; i < 32; ++i)
                y[i] = 32 + i < jo ? col[32 + i] : 0.f;
#pragma unroll
            for(int k = 0; k < 32; ++k)
#pragma unroll
                for(int i = 0; i < 32; ++i)
                    y[i] = fmaf(-sl[(32 + i) * LD + k], x[k], y[i]);
#pragma unroll
            for(int k = 0; k < 32; ++k)
#pragma unroll
                for(int i = k + 1; i < 32; ++i)
                    y[i] = fmaf(-sl[(32 + i) * LD + 32 + k], y[k], y[i]);
#pragma unroll
            for(int i = 0; i < 32; ++i)
                if(32 + i < jo)
                    col[32 + i] = y[i];
        }
    }
    __syncthreads();
}

// Two-level LU of one m x n FP32 matrix (PIVOT, split TF32): outer panels of LU2_JO columns
// factored by getrf_cta_dev (inner panel width JB, chunk cwi), the outer trailing update on
// tcgen05.  smem_raw: CtaLuSmem<float,NT,JB>::bytes(m, cwi, R) then the buffers of um.
template <int NT, int R, int JB>
__device__ __forceinline__ void getrf_cta2_dev(int m, int n, float* a, int lda, int* piv_out,
                                               int* info_out, int cw, int cwi,
                                               unsigned char* smem_raw, UmCtx& um,
                                               int* sinf)
{
    const int tid = threadIdx.x;
    const int mn = min(m, n);
    int inf = 0;
    for(int j0 = 0; j0 < mn; j0 += LU2_JO)
    {
        const int jo = min(LU2_JO, mn - j0);
        // 1. the outer panel (rows j0.., its jo columns) with the one-level kernel body
        getrf_cta_dev<float, NT, R, JB, 8, true, true>(m - j0, jo, a + ix(j0, j0, lda), lda,
                                                       piv_out + j0, sinf, cwi, true, smem_raw);
        __syncthreads();
        if(tid < jo)
            piv_out[j0 + tid] += j0;
        if(tid == 0 && inf == 0 && *sinf > 0)
            inf = *sinf + j0;
        __syncthreads();
        // 2. its row interchanges on the columns left and right of it, in LAPACK order
        for(int i = 0; i < jo; ++i)
        {
            const int p = piv_out[j0 + i] - 1, q = j0 + i;
            if(p != q)
                for(int c = tid; c < n - jo; c += NT)
                {
                    const int col = c < j0 ? c : c + jo;
                    const float t = a[ix(q, col, lda)];
                    a[ix(q, col, lda)] = a[ix(p, col, lda)];
                    a[ix(p, col, lda)] = t;
                }
            __syncthreads();
        }
        if(j0 + jo >= n)
            continue;
        // 3. U12 = L11^{-1} A12 (L11 staged in the space of the tcgen05 A operand)
        lu2_trsm<NT>(a, lda, j0, jo, n, um.ahi);
        // 4. A22 -= L21 U12 with K = jo
        umma_update_k64<NT>(a, lda, j0 + jo, j0, j0, jo, m - j0 - jo, j0 + jo, n, cw, um);
    }
    if(tid == 0)
        *info_out = um.failed ? INT_MIN : inf;
}

// 128-thread CTAs: 3 per SM, or LU_MIN_BLOCKS_128 when the panel fits the smaller register
// budget (FP32, or one row per thread); 256-thread CTAs: LU_MIN_BLOCKS, or one per SM for
// panels of more than 32 registers per thread (two rows of a 32-wide panel)
template <typename T, int NT, int R, int JB, int TN, bool PIVOT, bool TC = false,
          bool UM = false>
__global__ void __launch_bounds__(NT,
                                  UM ? (NT <= 128 ? 2 : 1)
                                  : NT <= 128 ? ((sizeof(T) == 4 || R == 1) ? LU_MIN_BLOCKS_128 : 3)
                                              : (R * JB > 32 ? 1 : LU_MIN_BLOCKS))
    getrf_cta_kernel(int m, int n, Batch<T> A, int lda, int* ipiv, int64_t strideP, int* info,
                     int cw, int fold, Gate gate)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int64_t b = blockIdx.x;
    if(gate.skip(b))
        return;
    if constexpr(!UM)
    {
        getrf_cta_dev<T, NT, R, JB, TN, PIVOT, TC>(m, n, A.at(b), lda,
                                                   PIVOT ? ipiv + b * strideP : nullptr,
                                                   info + b, cw, fold != 0, smem_raw);
    }
    else
    {
        // tcgen05 buffers after the LU's own shared memory; TMEM for one M-tile group
        __shared__ UmCtx um;
        uintptr_t p = reinterpret_cast<uintptr_t>(smem_raw) + CtaLuSmem<T, NT, JB>::bytes(m, cw, R);
        p = (p + 1023) & ~uintptr_t(1023);
        const int gmax = um_group_max<NT, JB>();
        const uint32_t ncols = umma::tmem_cols((uint32_t)(um_group<NT, JB>(cw) * cw));
        if(threadIdx.x == 0)
        {
            um.ahi = reinterpret_cast<float*>(p);
            um.alo = um.ahi + gmax * 128 * JB;
            um.bhi = um.alo + gmax * 128 * JB;
            um.blo = um.bhi + cw * JB;
            um.mbar = reinterpret_cast<uint64_t*>(um.blo + cw * JB);
            um.G = um_group<NT, JB>(cw);
            um.phase = 0;
            um.failed = 0;
            umma::mbar_init(um.mbar, 1);
        }
        if(threadIdx.x < 32)
            umma::tmem_alloc(reinterpret_cast<uint32_t*>(&um.tmem), ncols);
        umma::fence_before_sync();
        __syncthreads();
        umma::fence_after_sync();
        UmCtx mine = um; // per-thread copy: the phase and failure state advance in lockstep
        getrf_cta_dev<T, NT, R, JB, TN, PIVOT, TC, true>(m, n, A.at(b), lda, ipiv + b * strideP,
                                                         info + b, cw, false, smem_raw, &mine);
        umma::fence_before_sync();
        __syncthreads();
        if(threadIdx.x < 32)
            umma::tmem_free(mine.tmem, ncols);
    }
}

// Two-level FP32 LU (outer panels of 64 columns, K = 64 trailing updates on tcgen05): one CTA
// per matrix.  cw = outer update column chunk (<= 256), cwi = chunk of the inner panels.
template <int NT, int R, int JB>
__global__ void __launch_bounds__(NT, 1)
    getrf_cta2_kernel(int m, int n, Batch<float> A, int lda, int* ipiv, int64_t strideP,
                      int* info, int cw, int cwi, Gate gate)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int64_t b = blockIdx.x;
    if(gate.skip(b))
        return;
    __shared__ UmCtx um;
    __shared__ int sinf;
    uintptr_t p = reinterpret_cast<uintptr_t>(smem_raw) + CtaLuSmem<float, NT, JB>::bytes(m, cwi, R);
    p = (p + 1023) & ~uintptr_t(1023);
    const uint32_t ncols = umma::tmem_cols((uint32_t)cw);
    if(threadIdx.x == 0)
    {
        um.ahi = reinterpret_cast<float*>(p);
        um.alo = um.ahi + 128 * LU2_JO;
        um.bhi = um.alo + 128 * LU2_JO;
        um.blo = um.bhi + cw * LU2_JO;
        um.mbar = reinterpret_cast<uint64_t*>(um.blo + cw * LU2_JO);
        um.G = 1;
        um.phase = 0;
        um.failed = 0;
        umma::mbar_init(um.mbar, 1);
    }
    if(threadIdx.x < 32)
        umma::tmem_alloc(reinterpret_cast<uint32_t*>(&um.tmem), ncols);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    UmCtx mine = um;
    getrf_cta2_dev<NT, R, JB>(m, n, A.at(b), lda, ipiv + b * strideP, info + b, cw, cwi, smem_raw,
                              mine, &sinf);
    umma::fence_before_sync();
    __syncthreads();
    if(threadIdx.x < 32)
        umma::tmem_free(mine.tmem, ncols);
}

} // namespace rsb
