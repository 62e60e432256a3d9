// gather_tex.cu -- the texture copies that the fp16-feature stencil gather
// samples through the texture unit (mrp_params.gather_filter).
//
// The reference keeps its mip pyramid, TR levels and HG LUT in CUDA arrays
// behind hardware-filtered textures (Mip(i): trilinear, border addressing,
// core/volume.cu:1518-1521; TR_Mip(i): trilinear, clamp, :1656-1659;
// _HGLut: bilinear, clamp, :1414-1417; all with normalized coordinates) and
// SetupInputData samples them with tex3D / tex2D.  Here the builders write
// linear fp32 levels (the software gather and the FP32 form read those);
// these routines keep fp16 array copies of them for the texture path.  The
// features the texture path feeds are fp16 themselves, and fp16 texels
// halve the texture cache's footprint and filter at the unit's full rate.
// A level of edge n is stored z fastest, so the array's width is z -- the
// reference's texture coordinate x = pos.z + 0.5.
#include <cuda_fp16.h>

#include "kernels.h"
#include "dev_alloc.h"

namespace mrp {

namespace {
cudaError_t make_texture(cudaArray_t a, cudaTextureAddressMode mode, cudaTextureObject_t* t) {
    cudaResourceDesc res = {};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = a;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = mode;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    return cudaCreateTextureObject(t, &res, &td, nullptr);
}
cudaError_t make_surface(cudaArray_t a, cudaSurfaceObject_t* s) {
    cudaResourceDesc res = {};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = a;
    return cudaCreateSurfaceObject(s, &res);
}
cudaError_t alloc(int n, int depth, cudaTextureAddressMode mode, GtexLevel* L) {
    *L = GtexLevel{};
    cudaChannelFormatDesc desc = cudaCreateChannelDescHalf();
    cudaError_t e = dev_malloc_3d_array(&L->arr, &desc, make_cudaExtent(n, n, depth), cudaArraySurfaceLoadStore);
    if (e == cudaSuccess) e = make_texture(L->arr, mode, &L->tex);
    if (e == cudaSuccess) e = make_surface(L->arr, &L->surf);
    if (e != cudaSuccess) gtex_free(L);
    else L->n = n;
    return e;
}

// fp32 -> fp16 (round to nearest) into each level's array, one launch for up
// to kGtexMaxFill levels (blockIdx.y); 3D levels n^3 (x slowest, z fastest),
// 2D levels n x n (depth 0).
constexpr int kGtexMaxFill = 9;
struct FillTable {
    const float* src[kGtexMaxFill];
    cudaSurfaceObject_t surf[kGtexMaxFill];
    int n[kGtexMaxFill];
    int flat[kGtexMaxFill];   // 1: a 2D level
};
__global__ void __launch_bounds__(256) k_fill_half(const __grid_constant__ FillTable t) {
    const int L = blockIdx.y, n = t.n[L];
    const float* __restrict__ src = t.src[L];
    const size_t total = t.flat[L] ? (size_t)n * n : (size_t)n * n * n;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % n), y = (int)((i / n) % n), x = (int)(i / ((size_t)n * n));
        const unsigned short h = __half_as_ushort(__float2half_rn(__ldg(src + i)));
        if (t.flat[L]) surf2Dwrite(h, t.surf[L], z * (int)sizeof(h), y);
        else surf3Dwrite(h, t.surf[L], z * (int)sizeof(h), y, x);
    }
}
}  // namespace

cudaError_t gtex_alloc_level(int n, bool clamp, GtexLevel* L) {
    return alloc(n, n, clamp ? cudaAddressModeClamp : cudaAddressModeBorder, L);
}

cudaError_t gtex_alloc_lut(GtexLevel* L) {
    cudaError_t e = alloc(kLut, 0, cudaAddressModeClamp, L);
    L->flat = true;
    return e;
}

void gtex_free(GtexLevel* L) {
    if (L->surf) cudaDestroySurfaceObject(L->surf);
    if (L->tex) cudaDestroyTextureObject(L->tex);
    if (L->arr) dev_free_array(L->arr);
    *L = GtexLevel{};
}

cudaError_t gtex_fill(const GtexLevel* const* levels, const float* const* src, int count, int sms, cudaStream_t s) {
    for (int k = 0; k < count; k += kGtexMaxFill) {
        FillTable t{};
        const int m = count - k < kGtexMaxFill ? count - k : kGtexMaxFill;
        size_t most = 0;
        for (int i = 0; i < m; ++i) {
            const GtexLevel& L = *levels[k + i];
            if (!L.surf || !src[k + i]) return cudaErrorInvalidValue;
            t.src[i] = src[k + i];
            t.surf[i] = L.surf;
            t.n[i] = L.n;
            t.flat[i] = L.flat ? 1 : 0;
            const size_t texels = L.flat ? (size_t)L.n * L.n : (size_t)L.n * L.n * L.n;
            most = texels > most ? texels : most;
        }
        size_t want = (most + 255) / 256;
        const unsigned bx = (unsigned)(want < (size_t)sms * 8 ? want : (size_t)sms * 8);
        k_fill_half<<<dim3(bx > 0 ? bx : 1, m), 256, 0, s>>>(t);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

size_t gtex_level_bytes(int n) { return (size_t)n * n * n * sizeof(__half); }

}  // namespace mrp
