// vbatched_noalloc.cu -- the variable-size gesv for callers that cannot allocate.
//
// No counterpart in the reference.  rocsolver_dgesv_vbatched needs a little device scratch
// (its size-sorted work list and three work counters) and takes it from the handle's
// workspace, which the library allocates with cudaMalloc on first use.  Some callers cannot
// allow that: code that runs while a memory pool owns all device memory, allocation-free
// real-time loops, or plugins whose host framework forbids device allocations.  This entry
// point keeps that scratch in a fixed array in the library's own device memory instead, so
// it never allocates.
//
// Limits and sharing rules:
//   * at most VB_NOALLOC_MAX_BATCH members per call (larger batches get invalid_size);
//   * the array costs ~4 MiB on each GPU where the entry point has been called, until the
//     process exits.  With CUDA's lazy module loading (the default since CUDA 12.2) the driver
//     places it on the device when it first loads this module, at the first call's address
//     lookup: make the first call (a warm-up with batch_count > 0 will do) before a memory
//     pool claims the device's free memory, or that call returns internal_error;
//   * every call uses the same array: calls that overlap on the GPU (different streams, or
//     different handles on the same device without ordering) race and corrupt each other's
//     work lists; order them on one stream;
//   * the first call on each device looks up the array's device address (a CUDA runtime
//     query that may load the module, see above); make that first call before any stream
//     capture on the device.
// The contents left by the previous call need no clearing: the plan kernel rewrites the
// work list and resets the counters at the start of every call.
#include <mutex>

#include "handle.h"
#include "launch.h"
#include "logger.h"

namespace rsb {
namespace {

constexpr int VB_NOALLOC_MAX_BATCH = 1 << 20;
constexpr size_t VB_NOALLOC_BYTES =
    ((sizeof(int) * (size_t)VB_NOALLOC_MAX_BATCH + 255) & ~size_t(255)) + 256;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_vb_scratch[VB_NOALLOC_BYTES];

std::mutex g_mu;
void* g_addr[MAX_DEVICES] = {};

// device address of g_vb_scratch on the current device (looked up once per device)
rocblas_status scratch_address(void** out)
{
    int dev = -1;
    if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return rocblas_status_internal_error;
    std::lock_guard<std::mutex> lk(g_mu);
    if(!g_addr[dev])
    {
        void* p = nullptr;
        if(cudaGetSymbolAddress(&p, g_vb_scratch) != cudaSuccess || !p)
        {
            cudaGetLastError();
            return rocblas_status_internal_error;
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return rocblas_status_success;
}

} // namespace
} // namespace rsb

using namespace rsb;

extern "C" rocblas_status rocsolver_dgesv_vbatched_noalloc(
    rocblas_handle handle, const rocblas_int* n, const rocblas_int* nrhs, double* const A[],
    const rocblas_int* lda, rocblas_int* const ipiv[], double* const B[],
    const rocblas_int* ldb, rocblas_int* info, const rocblas_int max_n,
    const rocblas_int max_nrhs, const rocblas_int batch_count)
{
    RSB_LOG_TOP('d', "gesv_vbatched_noalloc", logging::arg("--max_n", max_n),
                logging::arg("--max_nrhs", max_nrhs), logging::arg("--batch_count", batch_count));
    if(!handle)
        return rocblas_status_invalid_handle;
    if(max_n < 0 || max_nrhs < 0 || batch_count < 0 || batch_count > VB_NOALLOC_MAX_BATCH)
        return rocblas_status_invalid_size;
    if(handle->querying)
        return ws_query(handle, 0);
    if(batch_count
       && (!n || !nrhs || !A || !lda || !ipiv || !B || !ldb || !info))
        return rocblas_status_invalid_pointer;
    if(batch_count == 0)
        return rocblas_status_success;
    void* scratch = nullptr;
    rocblas_status st = scratch_address(&scratch);
    if(st != rocblas_status_success)
        return st;
    return launch_vbatched<double>(handle->stream, 0, n, nrhs, A, lda, ipiv, B, ldb, info,
                                   max_n > 0 ? max_n : 1, max_nrhs, batch_count, scratch);
}
