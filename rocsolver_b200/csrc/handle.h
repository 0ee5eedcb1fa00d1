// handle.h -- internal view of rocblas_handle: {stream, workspace, size-query state}.
// Replaces the rocBLAS handle the reference borrows (library/src/include/rocblas.hpp,
// rocblas_device_malloc at lapack/roclapack_getrf_strided_batched.cpp:61-65).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "../../include/rocsolver.h"

struct _rocblas_handle
{
    cudaStream_t stream = 0;
    // workspace
    void* ws = nullptr;        // current device buffer (owned unless user_ws)
    size_t ws_size = 0;        // bytes allocated in ws
    size_t nominal = 32u << 20; // size reported by rocblas_get_device_memory_size
    bool managed = true;       // library grows the workspace on demand
    bool user_ws = false;      // ws belongs to the user (rocblas_set_workspace)
    int device = -1;           // device the owned buffer lives on
    // size query
    bool querying = false;
    size_t query_size = 0;
};

namespace rsb {

// Round a workspace request the way allocations are carved (256-byte aligned pieces).
inline size_t ws_round(size_t b) { return (b + 255) & ~size_t(255); }

// During a size query: record the request, return size_increased / size_unchanged.
rocblas_status ws_query(rocblas_handle h, size_t bytes);

// Make at least `bytes` of workspace available; returns nullptr via *out on bytes == 0.
// Returns memory_error when a user-fixed workspace is too small or cudaMalloc fails.
rocblas_status ws_get(rocblas_handle h, size_t bytes, void** out);

} // namespace rsb
