// handle.cpp -- rocBLAS handle shim mapped onto a CUDA stream plus a device workspace.
// Memory-model semantics follow clients/gtest/memory_model_gtest.cpp:54-170 of the
// reference (32 MiB nominal reservation; ROCBLAS_DEVICE_MEMORY_SIZE fixes the size;
// size queries report size_increased / size_unchanged without computing).
#include <cstdlib>
#include <cstring>
#include <new>

#include "handle.h"
#include "tuning.h"

namespace rsb {

rocblas_status ws_query(rocblas_handle h, size_t bytes)
{
    bytes = ws_round(bytes);
    if(bytes > h->query_size)
    {
        h->query_size = bytes;
        return rocblas_status_size_increased;
    }
    return rocblas_status_size_unchanged;
}

static void ws_release(rocblas_handle h)
{
    if(h->ws && !h->user_ws)
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if(h->device >= 0 && h->device != cur)
            cudaSetDevice(h->device);
        cudaFree(h->ws);
        if(h->device >= 0 && h->device != cur && cur >= 0)
            cudaSetDevice(cur);
    }
    h->ws = nullptr;
    h->ws_size = 0;
    h->user_ws = false;
}

rocblas_status ws_get(rocblas_handle h, size_t bytes, void** out)
{
    *out = nullptr;
    if(bytes == 0)
        return rocblas_status_success;
    bytes = ws_round(bytes);
    int dev = -1;
    if(cudaGetDevice(&dev) != cudaSuccess)
        return rocblas_status_internal_error;
    if(h->ws && h->ws_size >= bytes && (h->user_ws || h->device == dev))
    {
        *out = h->ws;
        return rocblas_status_success;
    }
    if(h->user_ws || !h->managed)
    {
        // fixed size: allocate once up to the fixed size, never grow beyond it
        if(h->user_ws || bytes > h->nominal)
            return rocblas_status_memory_error;
    }
    size_t want = bytes;
    if(!h->managed)
        want = h->nominal;
    // grow: the old buffer may still be in use by work queued on the stream
    if(h->ws)
    {
        cudaStreamSynchronize(h->stream);
        ws_release(h);
    }
    void* p = nullptr;
    if(cudaMalloc(&p, want) != cudaSuccess)
    {
        cudaGetLastError();
        return rocblas_status_memory_error;
    }
    h->ws = p;
    h->ws_size = want;
    h->device = dev;
    if(h->managed && want > h->nominal)
        h->nominal = want;
    *out = p;
    return rocblas_status_success;
}

} // namespace rsb

extern "C" {

rocblas_status rocblas_create_handle(rocblas_handle* handle)
{
    if(!handle)
        return rocblas_status_invalid_pointer;
    rsb::tuning_load_default_once();
    _rocblas_handle* h = new(std::nothrow) _rocblas_handle();
    if(!h)
        return rocblas_status_memory_error;
    const char* env = std::getenv("ROCBLAS_DEVICE_MEMORY_SIZE");
    if(env && *env)
    {
        char* end = nullptr;
        unsigned long long v = std::strtoull(env, &end, 10);
        if(end && *end == '\0' && v > 0)
        {
            h->nominal = (size_t)v;
            h->managed = false;
        }
    }
    *handle = h;
    return rocblas_status_success;
}

rocblas_status rocblas_destroy_handle(rocblas_handle handle)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    rsb::ws_release(handle);
    delete handle;
    return rocblas_status_success;
}

rocblas_status rocblas_set_stream(rocblas_handle handle, void* stream)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    handle->stream = (cudaStream_t)stream;
    return rocblas_status_success;
}

rocblas_status rocblas_get_stream(rocblas_handle handle, void** stream)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(!stream)
        return rocblas_status_invalid_pointer;
    *stream = (void*)handle->stream;
    return rocblas_status_success;
}

rocblas_status rocblas_start_device_memory_size_query(rocblas_handle handle)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(handle->querying)
        return rocblas_status_size_query_mismatch;
    handle->querying = true;
    handle->query_size = 0;
    return rocblas_status_success;
}

rocblas_status rocblas_stop_device_memory_size_query(rocblas_handle handle, size_t* size)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(!handle->querying)
        return rocblas_status_size_query_mismatch;
    if(!size)
        return rocblas_status_invalid_pointer;
    *size = handle->query_size;
    handle->querying = false;
    return rocblas_status_success;
}

int rocblas_is_device_memory_size_query(rocblas_handle handle)
{
    return handle && handle->querying ? 1 : 0;
}

int rocblas_is_managing_device_memory(rocblas_handle handle)
{
    return handle && handle->managed && !handle->user_ws ? 1 : 0;
}

rocblas_status rocblas_get_device_memory_size(rocblas_handle handle, size_t* size)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(!size)
        return rocblas_status_invalid_pointer;
    *size = handle->user_ws ? handle->ws_size : handle->nominal;
    return rocblas_status_success;
}

rocblas_status rocblas_set_device_memory_size(rocblas_handle handle, size_t size)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(handle->ws && !handle->user_ws)
        cudaStreamSynchronize(handle->stream);
    rsb::ws_release(handle);
    if(size == 0)
    {
        handle->managed = true;
        handle->nominal = 32u << 20;
        return rocblas_status_success;
    }
    handle->managed = false;
    handle->nominal = rsb::ws_round(size);
    return rocblas_status_success;
}

rocblas_status rocblas_set_workspace(rocblas_handle handle, void* addr, size_t size)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(handle->ws && !handle->user_ws)
        cudaStreamSynchronize(handle->stream);
    rsb::ws_release(handle);
    if(!addr || size == 0)
    {
        handle->managed = true;
        handle->nominal = 32u << 20;
        return rocblas_status_success;
    }
    handle->ws = addr;
    handle->ws_size = size;
    handle->user_ws = true;
    handle->managed = false;
    return rocblas_status_success;
}

#define RSB_VERSION_STRING "3.23.0-b200"

rocblas_status rocsolver_get_version_string(char* buf, size_t len)
{
    if(!buf)
        return rocblas_status_invalid_pointer;
    size_t need = std::strlen(RSB_VERSION_STRING) + 1;
    if(len < need)
        return rocblas_status_invalid_size;
    std::memcpy(buf, RSB_VERSION_STRING, need);
    return rocblas_status_success;
}

rocblas_status rocsolver_get_version_string_size(size_t* len)
{
    if(!len)
        return rocblas_status_invalid_pointer;
    *len = std::strlen(RSB_VERSION_STRING) + 1;
    return rocblas_status_success;
}

} // extern "C"
