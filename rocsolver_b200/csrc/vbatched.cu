// vbatched.cu -- variable-size batches (each member its own n, nrhs, lda, ldb) in ONE
// persistent launch.
//
// No counterpart in the reference (rocSOLVER batches are uniform in size).  Design:
//   1. plan kernel (one CTA): counting sort of the members by n, largest first, into a work
//      list in the workspace; members with n <= 32 go to a separate tail; work counters
//      are reset on the device, so the whole call is capturable in a CUDA graph;
//   2. persistent kernel: a grid of (SM count x resident CTAs) CTAs pulls work from the list
//      with atomicAdd.  A large member is factored and solved by the whole CTA (the same
//      device code as getrf/getrs); small members are taken eight at a time, one warp each,
//      with the register-resident warp LU + solve.  Largest-first ordering is the LPT rule:
//      the long factorisations start first and the short ones fill the tail.
// Per-member sizes live on the device; the host passes max_n / max_nrhs, which fix the
// kernel configuration and shared memory.  A member with n < 0, n > max_n, lda < n or
// (solve) ldb < n / nrhs < 0 / nrhs > max_nrhs gets info = -1 and is left untouched.
#include "handle.h"
#include "launch.h"
#include "logger.h"
#include "tuning.h"
#include "lu_cta.cuh"
#include "lu_small.cuh"
#include "trsv.cuh"

namespace rsb {

constexpr int VB_SMALL = 32;   // members with n <= VB_SMALL use the warp path
constexpr int VB_WARPS = 8;    // CTA = 8 warps = 256 threads

struct VbArgs
{
    int bc, max_n, max_nrhs, mode; // mode: 0 gesv, 1 getrf, 2 getrs
    const int* n;
    const int* nrhs;
    const int* lda;
    const int* ldb;
    int* const* ipiv;
    int* info;
    int* order;    // [bc]
    int* counters; // [0] big cursor, [1] small cursor, [2] number of big members
};

__global__ void __launch_bounds__(1024) vb_plan_kernel(VbArgs v)
{
    extern __shared__ int hist[]; // max_n + 2 buckets (n clamped; invalid -> bucket 0)
    const int nb = v.max_n + 2;
    for(int i = threadIdx.x; i < nb; i += blockDim.x)
        hist[i] = 0;
    __syncthreads();
    auto bucket = [&](int b) {
        const int n = v.n[b];
        if(n < 0 || n > v.max_n)
            return 0;
        return n + 1;
    };
    for(int b = threadIdx.x; b < v.bc; b += blockDim.x)
        atomicAdd(&hist[bucket(b)], 1);
    __syncthreads();
    if(threadIdx.x == 0)
    {
        // exclusive offsets in descending bucket order
        int acc = 0, nbig = 0;
        for(int k = nb - 1; k >= 0; --k)
        {
            const int c = hist[k];
            hist[k] = acc;
            acc += c;
            if(k - 1 > VB_SMALL)
                nbig = acc;
        }
        v.counters[0] = 0;
        v.counters[1] = nbig;
        v.counters[2] = nbig;
    }
    __syncthreads();
    for(int b = threadIdx.x; b < v.bc; b += blockDim.x)
        v.order[atomicAdd(&hist[bucket(b)], 1)] = b;
}

template <typename T>
__device__ __forceinline__ bool vb_valid(const VbArgs& v, int b)
{
    const int n = v.n[b];
    if(n < 0 || n > v.max_n || v.lda[b] < max(1, n))
        return false;
    if(v.mode != 1)
    {
        const int r = v.nrhs[b];
        if(r < 0 || r > v.max_nrhs || v.ldb[b] < max(1, n))
            return false;
    }
    return true;
}

template <typename T, int NT, int R, int JB, int TN>
__global__ void __launch_bounds__(NT, R * JB > 32 ? 1 : 2)
    vb_persistent_kernel(VbArgs v, T* const* A, T* const* B, int cw, int fold)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T srow[VB_WARPS][2][32];
    __shared__ int sown[VB_WARPS][32];
    __shared__ int task;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int nbig = v.counters[2];
    // ---- large members: the whole CTA per member
    for(;;)
    {
        if(tid == 0)
            task = atomicAdd(&v.counters[0], 1);
        __syncthreads();
        const int t = task;
        __syncthreads();
        if(t >= nbig)
            break;
        const int b = v.order[t];
        if(!vb_valid<T>(v, b))
        {
            if(tid == 0 && v.mode != 2)
                v.info[b] = -1;
            continue;
        }
        const int n = v.n[b];
        if(v.mode != 2)
        {
            // members up to 256 use the one-row-per-thread, 32-wide-panel configuration
            if(R > 1 && n <= NT)
                getrf_cta_dev<T, NT, 1, 32, TN, true>(n, n, A[b], v.lda[b], v.ipiv[b],
                                                      v.info + b, cw, fold != 0, smem_raw);
            else
                getrf_cta_dev<T, NT, R, JB, TN, true>(n, n, A[b], v.lda[b], v.ipiv[b],
                                                      v.info + b, cw, fold != 0, smem_raw);
            __syncthreads();
        }
        if(v.mode != 1 && (v.mode == 2 || v.info[b] == 0))
        {
            T* sdiag = reinterpret_cast<T*>(smem_raw);
            T* sb = sdiag + sweep_scratch<NT>();
            int* perm = reinterpret_cast<int*>(sb + (size_t)v.max_n * 4);
            getrs_dev<T, NT, 4>(0, n, v.nrhs[b], A[b], v.lda[b], v.ipiv[b], B[b], v.ldb[b], sb,
                                perm, sdiag);
        }
        __syncthreads();
    }
    // ---- small members: eight per CTA, one warp each
    for(;;)
    {
        if(tid == 0)
            task = atomicAdd(&v.counters[1], VB_WARPS);
        __syncthreads();
        const int t0 = task;
        __syncthreads();
        if(t0 >= v.bc)
            break;
        const int t = t0 + warp;
        if(t < v.bc)
        {
            const int b = v.order[t];
            if(!vb_valid<T>(v, b))
            {
                if((tid & 31) == 0 && v.mode != 2)
                    v.info[b] = -1;
            }
            else
            {
                const int n = v.n[b];
                if(v.mode == 2)
                {
                    // solve only: reuse the warp getrs through a one-member batch view
                    const int nr = v.nrhs[b];
                    const T* a = A[b];
                    T* x = B[b];
                    const int lane = tid & 31;
                    const int* piv = v.ipiv[b];
                    const int src = warp_perm_src(piv, n, lane);
                    const unsigned full = 0xffffffffu;
                    T r[32];
#pragma unroll
                    for(int j = 0; j < 32; ++j)
                        r[j] = (lane < n && j < n) ? a[ix(lane, j, v.lda[b])] : T(0);
                    for(int c = 0; c < nr; ++c)
                    {
                        T val = lane < n ? x[ix(src, c, v.ldb[b])] : T(0);
#pragma unroll
                        for(int k = 0; k < 32; ++k)
                            if(k < n)
                            {
                                T yk = __shfl_sync(full, val, k);
                                if(lane > k)
                                    val = fma(-r[k], yk, val);
                            }
#pragma unroll
                        for(int k = 31; k >= 0; --k)
                            if(k < n)
                            {
                                if(lane == k)
                                    val = val / r[k];
                                T xk = __shfl_sync(full, val, k);
                                if(lane < k)
                                    val = fma(-r[k], xk, val);
                            }
                        __syncwarp();
                        if(lane < n)
                            x[ix(lane, c, v.ldb[b])] = val;
                        __syncwarp();
                    }
                }
                else
                {
                    gesv_warp_dev<T, 32, 4>(n, v.mode == 0 ? v.nrhs[b] : 0, A[b], v.lda[b],
                                            v.ipiv[b], v.mode == 0 ? B[b] : nullptr,
                                            v.mode == 0 ? v.ldb[b] : 1, v.info + b, srow[warp],
                                            sown[warp]);
                }
            }
        }
        __syncthreads();
    }
}

size_t vbatched_workspace(int bc)
{
    return ws_round(sizeof(int) * (size_t)bc) + ws_round(sizeof(int) * 4);
}

static int sm_count()
{
    int dev = 0, c = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    return c;
}

// cw: trailing column chunk (0 = default), fold: interchange folding (see getrf_cta_dev),
// per_sm: CTAs launched per SM (0 = as many as fit).  *ran = false when the configuration
// cannot take this batch (too many rows, too much shared memory).
template <typename T, int NT, int R, int JB, int TN>
static rocblas_status run_vb(cudaStream_t s, VbArgs v, T* const* A, T* const* B, int cw,
                             int fold, int per_sm_req, bool* ran = nullptr)
{
    if(ran)
        *ran = false;
    if(v.max_n > NT * R)
        return rocblas_status_not_implemented;
    const int cwmax = sizeof(T) == 8 ? LU_CW_F64 : LU_CW_F32;
    const int nround = ((v.max_n + 31) / 32) * 32;
    if(cw <= 0)
        cw = cwmax;
    cw = ((cw + 31) / 32) * 32;
    if(cw > nround)
        cw = nround;
    size_t smem = CtaLuSmem<T, NT, JB>::bytes(v.max_n, cw, R);
    if(R > 1)
    {
        const size_t s1 = CtaLuSmem<T, NT, 32>::bytes(NT, cw, 1);
        if(s1 > smem)
            smem = s1;
    }
    const size_t solve = sizeof(T) * ((size_t)v.max_n * 4 + sweep_scratch<NT>())
                         + sizeof(int) * (size_t)v.max_n;
    if(solve > smem)
        smem = solve;
    if(smem > 227 * 1024)
        return rocblas_status_not_implemented;
    auto k = vb_persistent_kernel<T, NT, R, JB, TN>;
    if(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
       != cudaSuccess)
        return rocblas_status_internal_error;
    int per_sm = 1;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, smem) != cudaSuccess
       || per_sm < 1)
        per_sm = 1;
    if(per_sm_req > 0 && per_sm_req < per_sm)
        per_sm = per_sm_req;
    int grid = sm_count() * per_sm;
    if(grid > v.bc)
        grid = v.bc;
    if(ran)
        *ran = true;
    RSB_LOG_KERNEL("vb_persistent_kernel");
    k<<<grid, NT, smem, s>>>(v, A, B, cw, fold);
    return cudaGetLastError() == cudaSuccess ? rocblas_status_success
                                             : rocblas_status_internal_error;
}

template <typename T>
rocblas_status launch_vbatched(cudaStream_t s, int mode, const int* n, const int* nrhs,
                               T* const* A, const int* lda, int* const* ipiv, T* const* B,
                               const int* ldb, int* info, int max_n, int max_nrhs, int bc,
                               void* ws)
{
    if(max_n > MAX_CTA_ROWS || max_n > 4096)
        return rocblas_status_not_implemented;
    VbArgs v;
    v.bc = bc;
    v.max_n = max_n;
    v.max_nrhs = max_nrhs;
    v.mode = mode;
    v.n = n;
    v.nrhs = nrhs;
    v.lda = lda;
    v.ldb = ldb;
    v.ipiv = ipiv;
    v.info = info;
    v.order = static_cast<int*>(ws);
    v.counters = reinterpret_cast<int*>(static_cast<char*>(ws) + ws_round(sizeof(int) * bc));
    {
        RSB_LOG_KERNEL("vb_plan_kernel");
        vb_plan_kernel<<<1, 1024, sizeof(int) * (max_n + 2), s>>>(v);
    }
    if(cudaGetLastError() != cudaSuccess)
        return rocblas_status_internal_error;
    VbCfg c;
    if(tuned_vbatched(sizeof(T) == 8 ? 'd' : 's', max_n, &c) && c.nt == 256)
    {
        bool ran = false;
        rocblas_status st = rocblas_status_not_implemented;
        if(c.r == 1 && c.jb == 32)
            st = run_vb<T, 256, 1, 32, 8>(s, v, A, B, c.cw, c.fold, c.per_sm, &ran);
        else if(c.r == 2 && c.jb == 16)
            st = run_vb<T, 256, 2, 16, 8>(s, v, A, B, c.cw, c.fold, c.per_sm, &ran);
        else if(c.r == 2 && c.jb == 32)
            st = run_vb<T, 256, 2, 32, 8>(s, v, A, B, c.cw, c.fold, c.per_sm, &ran);
        else if(c.r == 4 && c.jb == 8)
            st = run_vb<T, 256, 4, 8, 4>(s, v, A, B, c.cw, c.fold, c.per_sm, &ran);
        else if(c.r == 4 && c.jb == 16)
            st = run_vb<T, 256, 4, 16, 8>(s, v, A, B, c.cw, c.fold, c.per_sm, &ran);
        else if(c.r == 8 && c.jb == 4)
            st = run_vb<T, 256, 8, 4, 4>(s, v, A, B, c.cw, c.fold, c.per_sm, &ran);
        if(ran)
            return st;
    }
    if(max_n <= 256)
        return run_vb<T, 256, 1, 32, 8>(s, v, A, B, 0, 0, 0);
    if(max_n <= 512)
        return run_vb<T, 256, 2, 16, 8>(s, v, A, B, 0, 0, 0);
    if(max_n <= 1024)
        return run_vb<T, 256, 4, 8, 4>(s, v, A, B, 0, 0, 0);
    return run_vb<T, 256, 8, 4, 4>(s, v, A, B, 0, 0, 0);
}

template rocblas_status launch_vbatched<float>(cudaStream_t, int, const int*, const int*,
                                               float* const*, const int*, int* const*,
                                               float* const*, const int*, int*, int, int, int,
                                               void*);
template rocblas_status launch_vbatched<double>(cudaStream_t, int, const int*, const int*,
                                                double* const*, const int*, int* const*,
                                                double* const*, const int*, int*, int, int, int,
                                                void*);

} // namespace rsb
