// common.cuh -- device helpers shared by the LU and Cholesky kernels.
//
// Layout conventions are the reference's (library/src/include/lib_host_helpers.hpp:21-24
// idx2D = i + j*lda; common/include/rocblas_utility.hpp:97-118 load_ptr_batch): member b of
// a strided batch starts at A + b*strideA, member b of a pointer-array batch is A[b].
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <float.h>
#include <limits.h>

namespace rsb {

// ---------------------------------------------------------------------------------------
// batch addressing: strided (ptrs == nullptr) or pointer array (ptrs != nullptr)
template <typename T>
struct Batch
{
    T* base;
    T* const* ptrs;
    int64_t stride;
    __device__ __forceinline__ T* at(int64_t b) const
    {
        return ptrs ? ptrs[b] : base + b * stride;
    }
};

template <typename T>
__host__ __device__ inline Batch<T> strided(T* p, int64_t s)
{
    return Batch<T>{p, nullptr, s};
}
template <typename T>
__host__ __device__ inline Batch<T> pointers(T* const* p)
{
    return Batch<T>{nullptr, p, 0};
}

// Per-member gate: with p == nullptr every member runs; otherwise member b runs only when
// (p[b] != 0) == run_if_nonzero.  Used to restrict a launch to a subset of the batch (the
// FP64 fallback of the mixed-precision solver) without compacting the batch on the host.
struct Gate
{
    const int* p;
    int run_if_nonzero;
    __device__ __forceinline__ bool skip(int64_t b) const
    {
        if(!p)
            return false;
        const bool nz = p[b] != 0;
        return run_if_nonzero ? !nz : nz;
    }
};
__host__ __device__ inline Gate no_gate()
{
    return Gate{nullptr, 0};
}

__device__ __forceinline__ size_t ix(int i, int j, int ld)
{
    return (size_t)i + (size_t)j * (size_t)ld;
}

// ---------------------------------------------------------------------------------------
// Bounds-checked build (nvcc -DRSB_BOUNDS_CHECK; python -m rocsolver_b200.build --checked).
// The reference's debug aid is ROCSOLVER_VERIFY_ASSUMPTIONS (library/src/include/
// lib_host_helpers.hpp:63-80).  Here every element access the factor and solve kernels make
// through RSB_AT(a, i, j, ld, m, n) checks 0 <= i < m <= ld and 0 <= j < n; a failed check
// does not trap: it counts the violation, records the first one (source line, i, j) and
// redirects the access to a scratch element, so the kernel runs to its end and the host
// reads the record with rocsolver_b200_bounds_check.  RSB_CHECK_PIV(p, n, line) checks a
// pivot index 1 <= p <= n the same way.  In the normal build both compile to the plain
// access.
#ifdef RSB_BOUNDS_CHECK
namespace bounds {
struct Record
{
    int count, line, i, j;
};
static __device__ Record g_rec;        // one per translation unit
static __device__ double g_scratch[4]; // target of redirected accesses
__device__ __forceinline__ void fail(int line, int i, int j)
{
    if(atomicAdd(&g_rec.count, 1) == 0)
    {
        g_rec.line = line;
        g_rec.i = i;
        g_rec.j = j;
    }
}
// host side: each translation unit registers a query of its record (bounds.cpp sums them)
typedef void (*QueryFn)(int* out4);
void register_query(QueryFn f);
static void query_tu(int* out4)
{
    Record r{};
    if(cudaMemcpyFromSymbol(&r, g_rec, sizeof(r)) != cudaSuccess)
    {
        cudaGetLastError();
        return;
    }
    const Record z{};
    cudaMemcpyToSymbol(g_rec, &z, sizeof(z));
    if(r.count && !out4[0])
    {
        out4[1] = r.line;
        out4[2] = r.i;
        out4[3] = r.j;
    }
    out4[0] += r.count;
}
static struct Registrar
{
    Registrar() { register_query(&query_tu); }
} g_registrar;
} // namespace bounds
template <typename T>
__device__ __forceinline__ T& at_checked(T* a, int i, int j, int ld, int m, int n, int line)
{
    if(i < 0 || i >= m || j < 0 || j >= n || ld < m)
    {
        bounds::fail(line, i, j);
        return *reinterpret_cast<T*>(bounds::g_scratch);
    }
    return a[ix(i, j, ld)];
}
#define RSB_AT(a, i, j, ld, m, n) (::rsb::at_checked((a), (i), (j), (ld), (m), (n), __LINE__))
#define RSB_CHECK_PIV(p, n, line)                                                            \
    do                                                                                       \
    {                                                                                        \
        if((p) < 1 || (p) > (n))                                                             \
            ::rsb::bounds::fail((line), (p), (n));                                           \
    } while(0)
#else
#define RSB_AT(a, i, j, ld, m, n) ((a)[::rsb::ix((i), (j), (ld))])
#define RSB_CHECK_PIV(p, n, line)                                                            \
    do                                                                                       \
    {                                                                                        \
    } while(0)
#endif

template <typename T>
struct Lim;
template <>
struct Lim<double>
{
    static __device__ __forceinline__ double sfmin() { return DBL_MIN; }
    // correctly rounded reciprocal (same value as 1.0 / x)
    static __device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
};
template <>
struct Lim<float>
{
    static __device__ __forceinline__ float sfmin() { return FLT_MIN; }
    static __device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
};

// ---------------------------------------------------------------------------------------
// Pivot keys.  LAPACK's idamax (and the reference's iamax,
// library/src/include/lapack_device_functions.hpp:680-740) returns the FIRST index of
// the largest |x|, scanning with a strict '>' so that a NaN never replaces the running
// maximum.  A tree reduction reproduces that sequential rule exactly when:
//   key(x) = bit pattern of |x| (monotone in |x| for non-negative IEEE values),
//   a NaN in the first candidate row (row k) gets the largest key (it can never be
//   replaced), a NaN elsewhere gets key 0 (it can never win against row k), and
//   ties on the key go to the smallest logical row index.
__device__ __forceinline__ uint64_t pivot_key(double x, bool first_row)
{
    uint64_t u = (uint64_t)__double_as_longlong(x) & 0x7fffffffffffffffull;
    if(u > 0x7ff0000000000000ull)
        u = first_row ? 0xffffffffffffffffull : 0ull;
    return u;
}
__device__ __forceinline__ uint32_t pivot_key(float x, bool first_row)
{
    uint32_t u = (uint32_t)__float_as_uint(x) & 0x7fffffffu;
    if(u > 0x7f800000u)
        u = first_row ? 0xffffffffu : 0u;
    return u;
}

template <typename T>
struct KeyOf;
template <>
struct KeyOf<double>
{
    using type = uint64_t;
};
template <>
struct KeyOf<float>
{
    using type = uint32_t;
};

// Warp-wide argmax over (key, row) pairs: largest key, then smallest row.  Lanes with
// valid == false do not take part.  Returns the winning row (INT_MAX if none is valid)
// and the winning key through *kout.  Uses redux.sync (3 for 64-bit keys, 2 for 32-bit).
__device__ __forceinline__ int warp_argmax(uint64_t key, int row, bool valid, uint64_t* kout)
{
    const unsigned full = 0xffffffffu;
    uint32_t hi = valid ? (uint32_t)(key >> 32) : 0u;
    uint32_t mhi = __reduce_max_sync(full, hi);
    uint32_t lo = (valid && hi == mhi) ? (uint32_t)key : 0u;
    uint32_t mlo = __reduce_max_sync(full, lo);
    bool match = valid && hi == mhi && (uint32_t)key == mlo;
    int r = (int)__reduce_min_sync(full, (unsigned)(match ? row : INT_MAX));
    *kout = ((uint64_t)mhi << 32) | mlo;
    return r;
}
__device__ __forceinline__ int warp_argmax(uint32_t key, int row, bool valid, uint32_t* kout)
{
    const unsigned full = 0xffffffffu;
    uint32_t k = valid ? key : 0u;
    uint32_t mk = __reduce_max_sync(full, k);
    bool match = valid && key == mk;
    int r = (int)__reduce_min_sync(full, (unsigned)(match ? row : INT_MAX));
    *kout = mk;
    return r;
}

// warp_argmax with the common case cut short: when a single lane holds the largest key
// (the high 32 bits of a 64-bit key already decide it almost always) its row comes from that
// lane by one shuffle; the full tie-breaking reductions run only when keys collide.  Same
// result as warp_argmax (largest key, smallest row on ties; INT_MAX if no lane is valid).
__device__ __forceinline__ int warp_argmax_fast(uint64_t key, int row, bool valid)
{
    const unsigned full = 0xffffffffu;
    const uint32_t hi = valid ? (uint32_t)(key >> 32) : 0u;
    const uint32_t mhi = __reduce_max_sync(full, hi);
    const unsigned mh = __ballot_sync(full, valid && hi == mhi);
    if(__popc(mh) == 1)
        return __shfl_sync(full, row, __ffs(mh) - 1);
    const bool inhi = valid && hi == mhi;
    const uint32_t mlo = __reduce_max_sync(full, inhi ? (uint32_t)key : 0u);
    const bool match = inhi && (uint32_t)key == mlo;
    const unsigned ml = __ballot_sync(full, match);
    if(__popc(ml) == 1)
        return __shfl_sync(full, row, __ffs(ml) - 1);
    return (int)__reduce_min_sync(full, (unsigned)(match ? row : INT_MAX));
}
__device__ __forceinline__ int warp_argmax_fast(uint32_t key, int row, bool valid)
{
    const unsigned full = 0xffffffffu;
    const uint32_t k = valid ? key : 0u;
    const uint32_t mk = __reduce_max_sync(full, k);
    const bool match = valid && key == mk;
    const unsigned mm = __ballot_sync(full, match);
    if(__popc(mm) == 1)
        return __shfl_sync(full, row, __ffs(mm) - 1);
    return (int)__reduce_min_sync(full, (unsigned)(match ? row : INT_MAX));
}

// LAPACK getf2 column scaling: multiply by the reciprocal when |pivot| >= sfmin,
// otherwise divide (dgetf2; the reference always multiplies,
// specialized/roclapack_getf2_specialized_kernels.hpp:96-99, which differs only for
// subnormal pivots).  A zero pivot leaves the column unscaled.
// (rcp: the correctly rounded reciprocal of piv, computed by the caller)
template <typename T>
__device__ __forceinline__ T getf2_scale(T x, T piv, T rcp)
{
    return piv == T(0) ? x : (fabs(piv) >= Lim<T>::sfmin() ? x * rcp : x / piv);
}

// ---------------------------------------------------------------------------------------
// Rolled register rows (LU panels): the active column is register 0 and a rank-1 update
// writes column c+1+i into register i.
// Candidate rows are published shifted by one (dst[i] = v[i+1], dst[JB-1] = 0; the pivot
// value itself goes to its own slot) with 16-byte vector stores, so that the rank-1
// update, which pairs element i+1 of the pivot row with register i, reads aligned vectors.
template <typename T, int JB>
__device__ __forceinline__ void store_row_shifted(T* dst, const T (&v)[JB])
{
    auto at = [&](int i) { return i < JB ? v[i] : T(0); };
    if constexpr(sizeof(T) == 8)
    {
#pragma unroll
        for(int i = 0; i < JB; i += 2)
            *reinterpret_cast<double2*>(dst + i) = make_double2(at(i + 1), at(i + 2));
    }
    else
    {
#pragma unroll
        for(int i = 0; i < JB; i += 4)
            *reinterpret_cast<float4*>(dst + i) =
                make_float4(at(i + 1), at(i + 2), at(i + 3), at(i + 4));
    }
}
// v[i] = fma(-l, row[i], v[i+1]) for i <= lim (and i < JB-1) with row read as aligned
// vectors.  Registers above lim hold columns outside the panel; they are left stale, in
// groups of 8 skipped by a branch that is uniform across the CTA (lim depends only on
// the column).
template <typename T, int JB>
__device__ __forceinline__ void update_shift(T (&v)[JB], T l, const T* row, int lim)
{
#pragma unroll
    for(int g = 0; g < JB; g += 8)
    {
        if(g > lim)
            break;
        if constexpr(sizeof(T) == 8)
        {
#pragma unroll
            for(int i = g; i < g + 8 && i < JB; i += 2)
            {
                const double2 t = *reinterpret_cast<const double2*>(row + i);
                if(i + 1 < JB)
                    v[i] = fma(-l, t.x, v[i + 1]);
                if(i + 2 < JB)
                    v[i + 1] = fma(-l, t.y, v[i + 2]);
            }
        }
        else
        {
#pragma unroll
            for(int i = g; i < g + 8 && i < JB; i += 4)
            {
                const float4 t = *reinterpret_cast<const float4*>(row + i);
                const float e[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
                for(int u = 0; u < 4; ++u)
                    if(i + u + 1 < JB)
                        v[i + u] = fmaf(-l, e[u], v[i + u + 1]);
            }
        }
    }
}

// Copy count elements into shared memory, store(e, load(e)) for e = threadIdx.x, +NT, ...,
// with U loads per thread issued before their stores so that their latencies overlap
// (a load feeding a shared-memory store otherwise waits for the previous store's load).
template <int NT, int U, typename L, typename S>
__device__ __forceinline__ void staged_copy(int count, L load, S store)
{
    using V = decltype(load(0));
    for(int e0 = threadIdx.x; e0 < count; e0 += U * NT)
    {
        V t[U];
#pragma unroll
        for(int u = 0; u < U; ++u)
        {
            const int e = e0 + u * NT;
            if(e < count)
                t[u] = load(e);
        }
#pragma unroll
        for(int u = 0; u < U; ++u)
        {
            const int e = e0 + u * NT;
            if(e < count)
                store(e, t[u]);
        }
    }
}

} // namespace rsb
