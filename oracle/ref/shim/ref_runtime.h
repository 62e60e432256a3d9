// ref_runtime.h -- host stand-ins for the CUDA runtime calls, arrays,
// surfaces and kernel launches that the reference's core/volume.cu uses, so
// that its volume builders (the CPU pyramid of Update, Update_TR with Fill_TR,
// Fill_Hg, Fill_BakeTR, GetHGLut, SetHDRI) run unmodified on the CPU for the
// checker build in oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY.  Force-included after ref_prelude.h by the
// `ref` target of oracle/Makefile for the volume harness.
//
// A cudaArray here is host memory, allocated when it is first bound, copied
// to or read (the reference's constructor asks for a 1024^3 array it never
// fills).  A texture bound to an array samples it in software
// (ref_prelude.h's tex3D / tex2D); a surface bound to an array is written by
// surf2Dwrite / surf3Dwrite.  A kernel launch `K<<<grid, block>>>(args)` is
// rewritten by the recipe into `ref_launch(grid, block, [&] { K(args); })`,
// which runs every thread of the grid on host threads, block by block (none
// of the kernels run this way uses shared memory, barriers or warp
// collectives).
#pragma once
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <functional>

enum cudaError_t { cudaSuccess = 0, cudaErrorInvalidValue = 1 };
typedef cudaError_t cudaError;
enum cudaMemcpyKind { cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2,
                      cudaMemcpyDeviceToDevice = 3, cudaMemcpyDefault = 4 };
#define cudaArraySurfaceLoadStore 0x02
#define cudaHostAllocMapped 0x02
#define cudaDeviceMapHost 0x08
#define cudaSurfaceType2D 0x02
#define cudaSurfaceType3D 0x03

struct cudaChannelFormatDesc { int x, y, z, w, f; };
template <class T> inline cudaChannelFormatDesc cudaCreateChannelDesc() {
    return cudaChannelFormatDesc{(int)(8 * sizeof(T)), 0, 0, 0, 0};
}
struct cudaExtent { size_t width, height, depth; };
inline cudaExtent make_cudaExtent(size_t w, size_t h, size_t d) { return cudaExtent{w, h, d}; }
struct cudaPitchedPtr { void* ptr; size_t pitch, xsize, ysize; };
inline cudaPitchedPtr make_cudaPitchedPtr(void* p, size_t pitch, size_t xs, size_t ys) {
    return cudaPitchedPtr{p, pitch, xs, ys};
}
struct cudaPos { size_t x, y, z; };

// Host-memory array: width is the fastest axis (the texture x); elem bytes
// per element (4 for float, 16 for float4).
struct cudaArray {
    size_t width = 0, height = 1, depth = 1, elem = 4;
    unsigned char* data = nullptr;
    unsigned char* mem() {
        if (!data) data = (unsigned char*)std::calloc(width * height * depth, elem);
        return data;
    }
    size_t bytes() const { return width * height * depth * elem; }
};
typedef cudaArray* cudaArray_t;
struct cudaMemcpy3DParms {
    cudaArray* srcArray; cudaPos srcPos; cudaPitchedPtr srcPtr;
    cudaArray* dstArray; cudaPos dstPos; cudaPitchedPtr dstPtr;
    cudaExtent extent; cudaMemcpyKind kind;
};

cudaError_t cudaMalloc3DArray(cudaArray** a, const cudaChannelFormatDesc* desc, cudaExtent e, unsigned flags = 0);
cudaError_t cudaMallocArray(cudaArray** a, const cudaChannelFormatDesc* desc, size_t w, size_t h = 0,
                            unsigned flags = 0);
cudaError_t cudaFreeArray(cudaArray* a);
cudaError_t cudaMemcpy3D(const cudaMemcpy3DParms* p);
cudaError_t cudaMemcpyToArray(cudaArray* dst, size_t wOffset, size_t hOffset, const void* src, size_t count,
                              cudaMemcpyKind kind);
cudaError_t cudaMalloc(void** p, size_t bytes);
template <class T> inline cudaError_t cudaMalloc(T** p, size_t bytes) { return cudaMalloc((void**)p, bytes); }
cudaError_t cudaFree(void* p);
cudaError_t cudaMemcpy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind);
cudaError_t cudaHostAlloc(void** p, size_t bytes, unsigned flags);
template <class T> inline cudaError_t cudaHostAlloc(T** p, size_t bytes, unsigned f) {
    return cudaHostAlloc((void**)p, bytes, f);
}
cudaError_t cudaHostGetDevicePointer(void** d, void* h, unsigned flags);
template <class T> inline cudaError_t cudaHostGetDevicePointer(T** d, void* h, unsigned f) {
    return cudaHostGetDevicePointer((void**)d, h, f);
}
cudaError_t cudaFreeHost(void* p);
cudaError_t cudaSetDeviceFlags(unsigned flags);
cudaError_t cudaDeviceSynchronize();
cudaError_t cudaGetLastError();
const char* cudaGetErrorString(cudaError_t e);
template <class T>
inline cudaError_t cudaMemcpyToSymbol(T& symbol, const void* src, size_t count, size_t offset = 0,
                                      cudaMemcpyKind = cudaMemcpyHostToDevice) {
    std::memcpy((unsigned char*)&symbol + offset, src, count);
    return cudaSuccess;
}

// texture binding: the texture samples the array's host memory
template <class T, int D, int M>
inline cudaError_t cudaBindTextureToArray(texture<T, D, M>& t, cudaArray* a, const cudaChannelFormatDesc& = {}) {
    if (!a) { t.data = nullptr; return cudaErrorInvalidValue; }
    t.data = (const T*)a->mem();
    t.nx = (int)a->width; t.ny = (int)a->height; t.nz = (int)a->depth;
    return cudaSuccess;
}

template <class T, int D = cudaSurfaceType2D>
struct surface {
    cudaArray* array = nullptr;
};
template <class T, int D>
inline cudaError_t cudaBindSurfaceToArray(surface<T, D>& s, cudaArray* a, const cudaChannelFormatDesc& = {}) {
    s.array = a;
    if (a) a->mem();   // allocated here, before a launch writes it from several threads
    return a ? cudaSuccess : cudaErrorInvalidValue;
}
// the value of the most recent surface write of this host thread (lets a
// harness run one thread of a kernel without binding a full-size array)
extern thread_local float ref_last_surface_value;
template <class T, int D>
inline void surf2Dwrite(float v, const surface<T, D>& s, int xbytes, int y) {
    ref_last_surface_value = v;
    if (!s.array) return;
    cudaArray* a = s.array;
    size_t x = (size_t)xbytes / sizeof(float);
    if (x < a->width && (size_t)y < a->height) ((float*)a->data)[(size_t)y * a->width + x] = v;
}
template <class T, int D>
inline void surf3Dwrite(float v, const surface<T, D>& s, int xbytes, int y, int z) {
    ref_last_surface_value = v;
    if (!s.array) return;
    cudaArray* a = s.array;
    size_t x = (size_t)xbytes / sizeof(float);
    if (x < a->width && (size_t)y < a->height && (size_t)z < a->depth)
        ((float*)a->data)[((size_t)z * a->height + y) * a->width + x] = v;
}

inline int atomicAdd(int* p, int v) { int o = *p; *p += v; return o; }

// Runs every thread of a grid: blocks are spread over host threads; the
// threads of one block run one after another on the block's host thread.
void ref_launch_blocks(dim3 grid, dim3 block, const std::function<void()>& body);
inline dim3 ref_dim3(dim3 d) { return d; }
inline dim3 ref_dim3(int d) { return dim3((unsigned)d); }
inline dim3 ref_dim3(unsigned d) { return dim3(d); }
template <class G, class B, class F>
inline void ref_launch(G grid, B block, F body) {
    ref_launch_blocks(ref_dim3(grid), ref_dim3(block), std::function<void()>(body));
}
