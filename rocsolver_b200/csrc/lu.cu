// lu.cu -- launchers for getrf / getrs / gesv and the Cholesky pair.
//
// Kernel selection by size replaces the reference's compile-time tuning tables
// (library/src/include/ideal_sizes.hpp:208-240 getrf, :166-180 potrf;
// roclapack_getf2.hpp:181-276 select_spkernel): the CTA LU configuration comes from the
// run-time tuning table (tuning.h) when it has an entry, else from the built-in choice.
#include <algorithm>

#include "chol.cuh"
#include "launch.h"
#include "logger.h"
#include "lu_cta.cuh"
#include "lu_small.cuh"
#include "trsv.cuh"
#include "tuning.h"

namespace rsb {

static inline rocblas_status launch_status()
{
    return cudaGetLastError() == cudaSuccess ? rocblas_status_success
                                             : rocblas_status_internal_error;
}

// Opt in to the dynamic shared memory a launch needs (static shared memory of the kernel
// counts against the same 48 KiB default, so the attribute is always set).
template <typename K>
static inline bool set_smem(K kernel, size_t bytes)
{
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bytes)
           == cudaSuccess;
}

__global__ void reset_info_kernel(int* info, int bc)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < bc)
        info[i] = 0;
}

rocblas_status launch_reset_info(cudaStream_t s, int* info, int bc)
{
    if(bc <= 0)
        return rocblas_status_success;
    reset_info_kernel<<<(bc + 255) / 256, 256, 0, s>>>(info, bc);
    return launch_status();
}

__global__ void reset_info2_kernel(int* a, int* b, int bc)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < bc)
    {
        a[i] = 0;
        b[i] = 0;
    }
}

rocblas_status launch_reset_info2(cudaStream_t s, int* a, int* b, int bc)
{
    if(bc <= 0)
        return rocblas_status_success;
    reset_info2_kernel<<<(bc + 255) / 256, 256, 0, s>>>(a, b, bc);
    return launch_status();
}

// ------------------------------------------------------------------------------ getrf
template <typename T, int NMAX, bool PIVOT>
static void run_getrf_warp(cudaStream_t s, int m, int n, Batch<T> A, int lda, int* ipiv,
                           int64_t sP, int* info, int bc, Gate g)
{
    dim3 grid((bc + SMALL_WPB - 1) / SMALL_WPB);
    RSB_LOG_KERNEL("getrf_warp_kernel");
    getrf_warp_kernel<T, NMAX, PIVOT><<<grid, 32 * SMALL_WPB, 0, s>>>(m, n, A, lda, ipiv, sP,
                                                                       info, bc, g);
}

// cw: trailing column chunk (multiple of 32); 0 picks the default (FP64: 64, FP32: 128 at
// most, so that two CTAs fit in an SM's shared memory).  *ran = false when the variant
// cannot take this size (more rows than threads x rows per thread, or too much shared
// memory): the caller then uses the built-in choice.
template <typename T, int NT, int R, int JB, bool PIVOT, bool TC = false, bool UM = false>
static rocblas_status run_getrf_cta(cudaStream_t s, int m, int n, Batch<T> A, int lda,
                                    int* ipiv, int64_t sP, int* info, int bc, Gate g, int cw,
                                    int fold, bool* ran = nullptr)
{
    if(ran)
        *ran = false;
    if(m > NT * R)
        return rocblas_status_not_implemented;
    const int cwmax = sizeof(T) == 8 ? LU_CW_F64 : LU_CW_F32;
    const int nround = ((n + 31) / 32) * 32;
    if(cw <= 0)
        cw = cwmax;
    cw = ((cw + 31) / 32) * 32;
    if(cw > nround)
        cw = nround;
    if(UM && cw > 256) // one MMA covers at most 256 columns
        cw = 256;
    size_t smem = CtaLuSmem<T, NT, JB>::bytes(m, cw, R);
    if constexpr(UM)
        smem += um_bytes<NT, JB>(cw);
    if(smem > 227 * 1024)
        return rocblas_status_not_implemented;
    auto k = getrf_cta_kernel<T, NT, R, JB, 8, PIVOT, TC, UM>;
    if(!set_smem(k, smem))
        return rocblas_status_internal_error;
    if(ran)
        *ran = true;
    RSB_LOG_KERNEL("getrf_cta_kernel");
    k<<<bc, NT, smem, s>>>(m, n, A, lda, ipiv, sP, info, cw, fold, g);
    return launch_status();
}

// two-level FP32 LU (outer panels of 64 columns, tcgen05 trailing updates with K = 64)
template <int NT, int R, int JB>
static rocblas_status run_getrf_cta2(cudaStream_t s, int m, int n, Batch<float> A, int lda,
                                     int* ipiv, int64_t sP, int* info, int bc, Gate g, int cw,
                                     bool* ran)
{
    *ran = false;
    if(m > NT * R)
        return rocblas_status_not_implemented;
    const int nround = ((n + 31) / 32) * 32;
    if(cw <= 0)
        cw = 128;
    cw = ((cw + 31) / 32) * 32;
    cw = std::min(std::min(cw, 256), std::max(nround, 32));
    const int cwi = LU2_JO;
    const size_t smem = CtaLuSmem<float, NT, JB>::bytes(m, cwi, R) + lu2_bytes(cw);
    if(smem > 227 * 1024)
        return rocblas_status_not_implemented;
    auto k = getrf_cta2_kernel<NT, R, JB>;
    if(!set_smem(k, smem))
        return rocblas_status_internal_error;
    *ran = true;
    RSB_LOG_KERNEL("getrf_cta2_kernel");
    k<<<bc, NT, smem, s>>>(m, n, A, lda, ipiv, sP, info, cw, cwi, g);
    return launch_status();
}

// the compiled CTA variants a tuning entry may name: (threads, rows per thread, panel width)
template <typename T, bool PIVOT, bool TC>
static rocblas_status run_getrf_tuned(const LuCfg& c, cudaStream_t s, int m, int n,
                                      Batch<T> A, int lda, int* ipiv, int64_t sP, int* info,
                                      int bc, Gate g, bool* ran)
{
    *ran = false;
    // fold = 2 selects the tcgen05 trailing update (FP32 split-TF32 variants, panel widths
    // that are multiples of 8)
    if constexpr(sizeof(T) == 4 && TC && PIVOT)
    {
        // fold = 3: two-level LU (outer panels of 64 columns on tcgen05)
        if(c.fold == 3)
        {
#define RSB_LU2_VARIANT(NT_, R_, JB_)                                                          \
            if(c.nt == NT_ && c.r == R_ && c.jb == JB_)                                        \
                return run_getrf_cta2<NT_, R_, JB_>(s, m, n, A, lda, ipiv, sP, info, bc, g, c.cw, \
                                                    ran);
            RSB_LU2_VARIANT(256, 2, 32)
            RSB_LU2_VARIANT(256, 2, 16)
            RSB_LU2_VARIANT(256, 4, 16)
            RSB_LU2_VARIANT(256, 4, 8)
            RSB_LU2_VARIANT(256, 8, 8)
#undef RSB_LU2_VARIANT
            return rocblas_status_not_implemented;
        }
        if(c.fold == 2)
        {
#define RSB_LU_UM_VARIANT(NT_, R_, JB_)                                                        \
            if(c.nt == NT_ && c.r == R_ && c.jb == JB_)                                        \
                return run_getrf_cta<T, NT_, R_, JB_, PIVOT, TC, true>(s, m, n, A, lda, ipiv, \
                                                                       sP, info, bc, g, c.cw, 0, \
                                                                       ran);
            RSB_LU_UM_VARIANT(128, 1, 32)
            RSB_LU_UM_VARIANT(128, 2, 32)
            RSB_LU_UM_VARIANT(256, 1, 32)
            RSB_LU_UM_VARIANT(256, 2, 32)
            RSB_LU_UM_VARIANT(256, 2, 16)
            RSB_LU_UM_VARIANT(256, 4, 16)
            RSB_LU_UM_VARIANT(256, 4, 8)
            RSB_LU_UM_VARIANT(256, 8, 8)
#undef RSB_LU_UM_VARIANT
            return rocblas_status_not_implemented;
        }
    }
#define RSB_LU_VARIANT(NT_, R_, JB_)                                                          \
    if(c.nt == NT_ && c.r == R_ && c.jb == JB_)                                                \
        return run_getrf_cta<T, NT_, R_, JB_, PIVOT, TC>(s, m, n, A, lda, ipiv, sP, info, bc, \
                                                         g, c.cw, c.fold, ran);
    RSB_LU_VARIANT(64, 1, 32)
    RSB_LU_VARIANT(128, 1, 32)
    RSB_LU_VARIANT(128, 2, 32)
    RSB_LU_VARIANT(128, 2, 16)
    RSB_LU_VARIANT(128, 4, 16)
    RSB_LU_VARIANT(256, 1, 32)
    RSB_LU_VARIANT(256, 2, 16)
    RSB_LU_VARIANT(256, 2, 32)
    RSB_LU_VARIANT(256, 4, 8)
    RSB_LU_VARIANT(256, 4, 16)
    RSB_LU_VARIANT(256, 8, 4)
    RSB_LU_VARIANT(256, 8, 8)
#undef RSB_LU_VARIANT
    return rocblas_status_not_implemented;
}

template <typename T, bool PIVOT, bool TC>
static rocblas_status getrf_dispatch(cudaStream_t s, int m, int n, Batch<T> A, int lda,
                                     int* ipiv, int64_t sP, int* info, int bc, Gate g)
{
    if(m <= 32 && n <= 32)
    {
        if(n <= 8)
            run_getrf_warp<T, 8, PIVOT>(s, m, n, A, lda, ipiv, sP, info, bc, g);
        else if(n <= 16)
            run_getrf_warp<T, 16, PIVOT>(s, m, n, A, lda, ipiv, sP, info, bc, g);
        else
            run_getrf_warp<T, 32, PIVOT>(s, m, n, A, lda, ipiv, sP, info, bc, g);
        return launch_status();
    }
    LuCfg c;
    const char prec = sizeof(T) == 8 ? 'd' : 's';
    if((TC && tuned_getrf('t', m, &c)) || tuned_getrf(prec, m, &c))
    {
        bool ran = false;
        const rocblas_status st =
            run_getrf_tuned<T, PIVOT, TC>(c, s, m, n, A, lda, ipiv, sP, info, bc, g, &ran);
        if(ran)
            return st;
    }
    // built-in choice (used when no tuning table is installed)
    if(m <= 64)
        return run_getrf_cta<T, 64, 1, 32, PIVOT, TC>(s, m, n, A, lda, ipiv, sP, info, bc,
                                                   g, 0, 0);
    if(m <= 128)
        return run_getrf_cta<T, 128, 1, 32, PIVOT, TC>(s, m, n, A, lda, ipiv, sP, info, bc,
                                                   g, 0, 0);
    // FP32: 128-thread CTAs with two rows per thread (three CTAs per SM); FP64 keeps
    // 256 threads (its two-row panel would not fit the register budget)
    if(sizeof(T) == 4 && m <= 256)
        return run_getrf_cta<T, 128, 2, 32, PIVOT, TC>(s, m, n, A, lda, ipiv, sP, info, bc,
                                                   g, 0, 0);
    if(m <= 256)
        return run_getrf_cta<T, 256, 1, 32, PIVOT, TC>(s, m, n, A, lda, ipiv, sP, info, bc,
                                                   g, 0, 0);
    if(m <= 512)
        return run_getrf_cta<T, 256, 2, 16, PIVOT, TC>(s, m, n, A, lda, ipiv, sP, info, bc,
                                                   g, 0, 0);
    if(m <= 1024)
        return run_getrf_cta<T, 256, 4, 8, PIVOT, TC>(s, m, n, A, lda, ipiv, sP, info, bc,
                                                   g, 0, 0);
    if(m <= MAX_CTA_ROWS)
        return run_getrf_cta<T, 256, 8, 4, PIVOT, TC>(s, m, n, A, lda, ipiv, sP, info, bc,
                                                   g, 0, 0);
    return rocblas_status_not_implemented;
}

template <typename T>
rocblas_status launch_getrf(cudaStream_t s, int m, int n, Batch<T> A, int lda, int* ipiv,
                            int64_t sP, int* info, int bc, bool pivot, Gate g, bool tc)
{
    if constexpr(sizeof(T) == 4)
        if(tc && pivot)
            return getrf_dispatch<T, true, true>(s, m, n, A, lda, ipiv, sP, info, bc, g);
    return pivot ? getrf_dispatch<T, true, false>(s, m, n, A, lda, ipiv, sP, info, bc, g)
                 : getrf_dispatch<T, false, false>(s, m, n, A, lda, ipiv, sP, info, bc, g);
}

// ------------------------------------------------------------------------------ getrs
template <typename T, int NMAX, int NRC>
static void run_getrs_warp(cudaStream_t s, int trans, int n, int nrhs, Batch<T> A, int lda,
                           const int* ipiv, int64_t sP, Batch<T> B, int ldb, const int* skip,
                           int bc, Gate g)
{
    const int64_t tasks = (int64_t)bc * ((nrhs + NRC - 1) / NRC);
    dim3 grid((unsigned)((tasks + SMALL_WPB - 1) / SMALL_WPB));
    RSB_LOG_KERNEL("getrs_warp_kernel");
    getrs_warp_kernel<T, NMAX, NRC><<<grid, 32 * SMALL_WPB, 0, s>>>(trans, n, nrhs, A, lda, ipiv,
                                                                     sP, B, ldb, skip, bc, g);
}

template <typename T, int NMAX>
static void getrs_warp_nrc(cudaStream_t s, int trans, int n, int nrhs, Batch<T> A, int lda,
                           const int* ipiv, int64_t sP, Batch<T> B, int ldb, const int* skip,
                           int bc, Gate g)
{
    if(nrhs == 1)
        run_getrs_warp<T, NMAX, 1>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc, g);
    else
        run_getrs_warp<T, NMAX, 4>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc, g);
}

template <typename T, int NT, int NRC>
static rocblas_status run_getrs_cta_nt(cudaStream_t s, int trans, int n, int nrhs, Batch<T> A,
                                       int lda, const int* ipiv, int64_t sP, Batch<T> B,
                                       int ldb, const int* skip, int bc, Gate g)
{
    const size_t smem =
        sizeof(T) * ((size_t)n * NRC + sweep_scratch<NT>()) + sizeof(int) * (size_t)n;
    auto k = getrs_cta_kernel<T, NT, NRC>;
    if(!set_smem(k, smem))
        return rocblas_status_internal_error;
    const int64_t groups = (nrhs + NRC - 1) / NRC;
    RSB_LOG_KERNEL("getrs_cta_kernel");
    k<<<(unsigned)(bc * groups), NT, smem, s>>>(trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip,
                                                g);
    return launch_status();
}

// CTA size follows n: one thread per row for the off-diagonal updates
template <typename T, int NRC>
static rocblas_status run_getrs_cta(cudaStream_t s, int trans, int n, int nrhs, Batch<T> A,
                                    int lda, const int* ipiv, int64_t sP, Batch<T> B, int ldb,
                                    const int* skip, int bc, Gate g)
{
    if(n <= 64)
        return run_getrs_cta_nt<T, 64, NRC>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip,
                                            bc, g);
    if(n <= 128)
        return run_getrs_cta_nt<T, 128, NRC>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip,
                                             bc, g);
    return run_getrs_cta_nt<T, 256, NRC>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc,
                                         g);
}

template <typename T>
rocblas_status launch_getrs(cudaStream_t s, int trans, int n, int nrhs, Batch<T> A, int lda,
                            const int* ipiv, int64_t sP, Batch<T> B, int ldb, const int* skip,
                            int bc, Gate g)
{
    if(n <= 8)
        getrs_warp_nrc<T, 8>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc, g);
    else if(n <= 16)
        getrs_warp_nrc<T, 16>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc, g);
    else if(n <= 32)
        getrs_warp_nrc<T, 32>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc, g);
    else if(n <= 4096)
        return nrhs == 1
                   ? run_getrs_cta<T, 1>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc, g)
                   : run_getrs_cta<T, 4>(s, trans, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc, g);
    else
        return rocblas_status_not_implemented;
    return launch_status();
}

// ------------------------------------------------------------------------------ gesv
template <typename T, int NMAX>
static void run_gesv_warp(cudaStream_t s, int n, int nrhs, Batch<T> A, int lda, int* ipiv,
                          int64_t sP, Batch<T> B, int ldb, int* info, int bc)
{
    dim3 grid((bc + SMALL_WPB - 1) / SMALL_WPB);
    RSB_LOG_KERNEL("gesv_warp_kernel");
    if(nrhs == 1)
        gesv_warp_kernel<T, NMAX, 1><<<grid, 32 * SMALL_WPB, 0, s>>>(n, nrhs, A, lda, ipiv, sP,
                                                                      B, ldb, info, bc);
    else
        gesv_warp_kernel<T, NMAX, 4><<<grid, 32 * SMALL_WPB, 0, s>>>(n, nrhs, A, lda, ipiv, sP,
                                                                      B, ldb, info, bc);
}

template <typename T>
rocblas_status launch_gesv(cudaStream_t s, int n, int nrhs, Batch<T> A, int lda, int* ipiv,
                           int64_t sP, Batch<T> B, int ldb, int* info, int bc)
{
    if(n <= 32)
    {
        if(n <= 8)
            run_gesv_warp<T, 8>(s, n, nrhs, A, lda, ipiv, sP, B, ldb, info, bc);
        else if(n <= 16)
            run_gesv_warp<T, 16>(s, n, nrhs, A, lda, ipiv, sP, B, ldb, info, bc);
        else
            run_gesv_warp<T, 32>(s, n, nrhs, A, lda, ipiv, sP, B, ldb, info, bc);
        return launch_status();
    }
    rocblas_status st = launch_getrf<T>(s, n, n, A, lda, ipiv, sP, info, bc, true);
    if(st != rocblas_status_success)
        return st;
    return launch_getrs<T>(s, 0, n, nrhs, A, lda, ipiv, sP, B, ldb, info, bc);
}

// ------------------------------------------------------------------------------ potrf
template <typename T, int NT, int R, int JB, int TN>
static rocblas_status run_potrf(cudaStream_t s, int upper, int n, Batch<T> A, int lda,
                                int* info, int bc)
{
    size_t smem = sizeof(T) * 2 * JB;
    if(n > JB)
        smem += sizeof(T) * (size_t)R * NT * (JB + 1);
    auto k = potrf_cta_kernel<T, NT, R, JB, TN>;
    if(!set_smem(k, smem))
        return rocblas_status_internal_error;
    RSB_LOG_KERNEL("potrf_cta_kernel");
    k<<<bc, NT, smem, s>>>(upper, n, A, lda, info);
    return launch_status();
}

template <typename T, int N>
static rocblas_status run_potrf_reg(cudaStream_t s, int upper, int n, Batch<T> A, int lda,
                                    int* info, int bc)
{
    RSB_LOG_KERNEL("potrf_reg_kernel");
    potrf_reg_kernel<T, N><<<bc, N, 0, s>>>(upper, n, A, lda, info);
    return launch_status();
}

template <typename T>
rocblas_status launch_potrf(cudaStream_t s, int upper, int n, Batch<T> A, int lda, int* info,
                            int bc)
{
    if(n <= 32)
        return run_potrf_reg<T, 32>(s, upper, n, A, lda, info, bc);
    if(n <= 64)
        return run_potrf_reg<T, 64>(s, upper, n, A, lda, info, bc);
    if(n <= 256)
        return run_potrf<T, 256, 1, 32, 8>(s, upper, n, A, lda, info, bc);
    if(n <= 512)
        return run_potrf<T, 256, 2, 16, 8>(s, upper, n, A, lda, info, bc);
    if(n <= 1024)
        return run_potrf<T, 256, 4, 8, 4>(s, upper, n, A, lda, info, bc);
    if(n <= MAX_CTA_ROWS)
        return run_potrf<T, 256, 8, 4, 4>(s, upper, n, A, lda, info, bc);
    return rocblas_status_not_implemented;
}

template <typename T, int NT, int NRC>
static rocblas_status run_potrs_nt(cudaStream_t s, int upper, int n, int nrhs, Batch<T> A,
                                   int lda, Batch<T> B, int ldb, const int* skip, int bc)
{
    const size_t smem = sizeof(T) * ((size_t)n * NRC + sweep_scratch<NT>());
    auto k = potrs_cta_kernel<T, NT, NRC>;
    if(!set_smem(k, smem))
        return rocblas_status_internal_error;
    const int64_t groups = (nrhs + NRC - 1) / NRC;
    RSB_LOG_KERNEL("potrs_cta_kernel");
    k<<<(unsigned)(bc * groups), NT, smem, s>>>(upper, n, nrhs, A, lda, B, ldb, skip);
    return launch_status();
}

template <typename T, int N, int NRC>
static rocblas_status run_potrs_small(cudaStream_t s, int upper, int n, int nrhs, Batch<T> A,
                                      int lda, Batch<T> B, int ldb, const int* skip, int bc)
{
    const int64_t groups = (nrhs + NRC - 1) / NRC;
    RSB_LOG_KERNEL("potrs_small_kernel");
    potrs_small_kernel<T, N, NRC>
        <<<(unsigned)(bc * groups), N, 0, s>>>(upper, n, nrhs, A, lda, B, ldb, skip);
    return launch_status();
}

template <typename T, int NRC>
static rocblas_status run_potrs(cudaStream_t s, int upper, int n, int nrhs, Batch<T> A,
                                int lda, Batch<T> B, int ldb, const int* skip, int bc)
{
    if(n <= 32)
        return run_potrs_small<T, 32, NRC>(s, upper, n, nrhs, A, lda, B, ldb, skip, bc);
    if(n <= 64)
        return run_potrs_small<T, 64, NRC>(s, upper, n, nrhs, A, lda, B, ldb, skip, bc);
    if(n <= 128)
        return run_potrs_nt<T, 128, NRC>(s, upper, n, nrhs, A, lda, B, ldb, skip, bc);
    return run_potrs_nt<T, 256, NRC>(s, upper, n, nrhs, A, lda, B, ldb, skip, bc);
}

template <typename T>
rocblas_status launch_potrs(cudaStream_t s, int upper, int n, int nrhs, Batch<T> A, int lda,
                            Batch<T> B, int ldb, const int* skip, int bc)
{
    if(n > 4096)
        return rocblas_status_not_implemented;
    return nrhs == 1 ? run_potrs<T, 1>(s, upper, n, nrhs, A, lda, B, ldb, skip, bc)
                     : run_potrs<T, 4>(s, upper, n, nrhs, A, lda, B, ldb, skip, bc);
}

// Solve with many right-hand sides (getri's n columns of the identity): 32 columns per CTA
// through shared memory for 32 < n <= 512, so that each CTA's pass over the factors (and its
// diagonal-block inversions) serves 32 columns instead of 4; otherwise launch_getrs.
template <typename T>
rocblas_status launch_getrs_many(cudaStream_t s, int n, int nrhs, Batch<T> A, int lda,
                                 const int* ipiv, int64_t sP, Batch<T> B, int ldb,
                                 const int* skip, int bc)
{
    if(n <= 32 || n > 512 || nrhs < 32)
        return launch_getrs<T>(s, 0, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc, no_gate());
    return run_getrs_cta<T, 32>(s, 0, n, nrhs, A, lda, ipiv, sP, B, ldb, skip, bc, no_gate());
}

// ------------------------------------------------------------------------------ instances
#define RSB_INST(T)                                                                          \
    template rocblas_status launch_getrf<T>(cudaStream_t, int, int, Batch<T>, int, int*,   \
                                            int64_t, int*, int, bool, Gate, bool);         \
    template rocblas_status launch_getrs<T>(cudaStream_t, int, int, int, Batch<T>, int,    \
                                            const int*, int64_t, Batch<T>, int, const int*, \
                                            int, Gate);                                    \
    template rocblas_status launch_gesv<T>(cudaStream_t, int, int, Batch<T>, int, int*,    \
                                           int64_t, Batch<T>, int, int*, int);             \
    template rocblas_status launch_potrf<T>(cudaStream_t, int, int, Batch<T>, int, int*,   \
                                            int);                                          \
    template rocblas_status launch_potrs<T>(cudaStream_t, int, int, int, Batch<T>, int,    \
                                            Batch<T>, int, const int*, int);               \
    template rocblas_status launch_getrs_many<T>(cudaStream_t, int, int, Batch<T>, int,    \
                                                 const int*, int64_t, Batch<T>, int,       \
                                                 const int*, int);
RSB_INST(float)
RSB_INST(double)

} // namespace rsb
