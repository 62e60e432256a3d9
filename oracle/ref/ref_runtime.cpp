// ref_runtime.cpp -- definitions behind shim/ref_runtime.h: CUDA arrays as
// host memory, host copies for the runtime's copy calls, and the launcher
// that runs a grid's threads on host threads.  TEST INFRASTRUCTURE ONLY
// (the volume harness of the CPU checker build in oracle/_ref/).
#include <atomic>
#include <thread>
#include <vector>

thread_local float ref_last_surface_value = 0.0f;

cudaError_t cudaMalloc3DArray(cudaArray** a, const cudaChannelFormatDesc* desc, cudaExtent e, unsigned) {
    cudaArray* r = new cudaArray;
    r->width = e.width;
    r->height = e.height ? e.height : 1;
    r->depth = e.depth ? e.depth : 1;
    r->elem = desc && desc->x > 0 ? (size_t)desc->x / 8 : 4;
    *a = r;
    return cudaSuccess;
}
cudaError_t cudaMallocArray(cudaArray** a, const cudaChannelFormatDesc* desc, size_t w, size_t h, unsigned f) {
    return cudaMalloc3DArray(a, desc, cudaExtent{w, h ? h : 1, 1}, f);
}
cudaError_t cudaFreeArray(cudaArray* a) {
    if (a) {
        std::free(a->data);
        delete a;
    }
    return cudaSuccess;
}
cudaError_t cudaMemcpy3D(const cudaMemcpy3DParms* p) {
    // host (pitched) -> array, the only direction core/volume.cu uses; a
    // null destination (an array the reference never allocated) is refused
    if (!p->dstArray || !p->srcPtr.ptr) return cudaErrorInvalidValue;
    cudaArray* a = p->dstArray;
    size_t row = p->extent.width * a->elem;
    for (size_t z = 0; z < p->extent.depth; ++z)
        for (size_t y = 0; y < p->extent.height; ++y)
            std::memcpy(a->mem() + ((z * a->height + y) * a->width) * a->elem,
                        (const unsigned char*)p->srcPtr.ptr + (z * p->srcPtr.ysize + y) * p->srcPtr.pitch, row);
    return cudaSuccess;
}
cudaError_t cudaMemcpyToArray(cudaArray* dst, size_t wOffset, size_t hOffset, const void* src, size_t count,
                              cudaMemcpyKind) {
    if (!dst) return cudaErrorInvalidValue;
    size_t off = (hOffset * dst->width + wOffset) * dst->elem;
    if (off + count > dst->bytes()) return cudaErrorInvalidValue;
    std::memcpy(dst->mem() + off, src, count);
    return cudaSuccess;
}
cudaError_t cudaMalloc(void** p, size_t bytes) {
    *p = std::calloc(bytes ? bytes : 1, 1);
    return *p ? cudaSuccess : cudaErrorInvalidValue;
}
cudaError_t cudaFree(void* p) {
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void* dst, const void* src, size_t bytes, cudaMemcpyKind) {
    std::memcpy(dst, src, bytes);
    return cudaSuccess;
}
cudaError_t cudaHostAlloc(void** p, size_t bytes, unsigned) { return cudaMalloc(p, bytes); }
cudaError_t cudaHostGetDevicePointer(void** d, void* h, unsigned) {
    *d = h;
    return cudaSuccess;
}
cudaError_t cudaFreeHost(void* p) { return cudaFree(p); }
cudaError_t cudaSetDeviceFlags(unsigned) { return cudaSuccess; }
cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
cudaError_t cudaGetLastError() { return cudaSuccess; }
const char* cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "invalid value"; }

void ref_launch_blocks(dim3 grid, dim3 block, const std::function<void()>& body) {
    const unsigned long long nblocks = (unsigned long long)grid.x * grid.y * grid.z;
    std::atomic<unsigned long long> next{0};
    unsigned nthreads = std::max(1u, std::thread::hardware_concurrency());
    auto worker = [&] {
        blockDim = block;
        gridDim = grid;
        for (;;) {
            unsigned long long b = next.fetch_add(1);
            if (b >= nblocks) break;
            blockIdx = uint3{(unsigned)(b % grid.x), (unsigned)((b / grid.x) % grid.y), (unsigned)(b / grid.x / grid.y)};
            for (unsigned tz = 0; tz < block.z; ++tz)
                for (unsigned ty = 0; ty < block.y; ++ty)
                    for (unsigned tx = 0; tx < block.x; ++tx) {
                        threadIdx = uint3{tx, ty, tz};
                        body();
                    }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned i = 0; i < nthreads; ++i) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
}
