// dev_alloc.h -- the library's only route to CUDA memory allocation.
//
// Every device, stream-ordered and pinned-host allocation (and every free)
// made by libmrpnn_b200 goes through these wrappers, which count the calls.
// mrp_debug_alloc_calls() exposes the count, so a caller or a test can check
// that an entry point which promises to allocate nothing (for instance
// mrp_predict_features_noalloc) made no allocation call, including one that
// was freed again before it returned.
#pragma once
#include <atomic>
#include <cstddef>

#include <cuda_runtime.h>

namespace mrp {

extern std::atomic<unsigned long long> g_alloc_calls;

template <class T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
    g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
    return cudaMalloc((void**)p, bytes);
}
template <class T>
inline cudaError_t dev_malloc_async(T** p, size_t bytes, cudaStream_t s) {
    g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
    return cudaMallocAsync((void**)p, bytes, s);
}
template <class T>
inline cudaError_t host_malloc_pinned(T** p, size_t bytes) {
    g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
    return cudaMallocHost((void**)p, bytes);
}
inline cudaError_t dev_free(void* p) {
    g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
    return cudaFree(p);
}
inline cudaError_t dev_free_async(void* p, cudaStream_t s) {
    g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
    return cudaFreeAsync(p, s);
}
inline cudaError_t dev_malloc_3d_array(cudaArray_t* a, const cudaChannelFormatDesc* desc, cudaExtent e,
                                       unsigned flags = 0) {
    g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
    return cudaMalloc3DArray(a, desc, e, flags);
}
inline cudaError_t dev_free_array(cudaArray_t a) {
    g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
    return cudaFreeArray(a);
}
inline cudaError_t host_free_pinned(void* p) {
    g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
    return cudaFreeHost(p);
}

}  // namespace mrp
