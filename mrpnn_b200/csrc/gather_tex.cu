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
// The (mip L, TR L - 1) pair levels, L = 1..7 (edge n = 256 >> L for both):
// half2 texels on a grid padded by one texel per side, read with clamp
// addressing and unnormalized coordinates.  The padding holds density 0
// (the mip's border value) and the TR level's edge texel (its clamp value),
// so one trilinear fetch of the pair returns what the mip's border-mode and
// the TR level's clamp-mode fetches return at the same point, anywhere.
struct PairTable {
    const float* mip[kGtexPairs];
    const float* tr[kGtexPairs];
    cudaSurfaceObject_t surf[kGtexPairs];
    int n[kGtexPairs];
};
__global__ void __launch_bounds__(256) k_fill_pairs(const __grid_constant__ PairTable t) {
    const int L = blockIdx.y, n = t.n[L], P = n + 2;
    if (n == 0) return;
    const size_t total = (size_t)P * P * P;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int zp = (int)(i % P), yp = (int)((i / P) % P), xp = (int)(i / ((size_t)P * P));
        const int x = xp - 1, y = yp - 1, z = zp - 1;
        const bool in = (unsigned)x < (unsigned)n && (unsigned)y < (unsigned)n && (unsigned)z < (unsigned)n;
        const int cx = min(max(x, 0), n - 1), cy = min(max(y, 0), n - 1), cz = min(max(z, 0), n - 1);
        const size_t c = ((size_t)cx * n + cy) * n + cz;
        const float d = in ? __ldg(t.mip[L] + c) : 0.0f;
        const __half2 h = __floats2half2_rn(d, __ldg(t.tr[L] + c));
        surf3Dwrite(*reinterpret_cast<const unsigned*>(&h), t.surf[L], zp * 4, yp, xp);
    }
}
}  // namespace

cudaError_t gtex_alloc_pair(int n, GtexLevel* L) {
    *L = GtexLevel{};
    const int P = n + 2;
    cudaChannelFormatDesc desc = cudaCreateChannelDescHalf2();
    cudaError_t e = dev_malloc_3d_array(&L->arr, &desc, make_cudaExtent(P, P, P), cudaArraySurfaceLoadStore);
    if (e == cudaSuccess) {
        cudaResourceDesc res = {};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = L->arr;
        cudaTextureDesc td = {};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        e = cudaCreateTextureObject(&L->tex, &res, &td, nullptr);
    }
    if (e == cudaSuccess) e = make_surface(L->arr, &L->surf);
    if (e != cudaSuccess) gtex_free(L);
    else L->n = n;
    return e;
}

cudaError_t gtex_fill_pairs(const GtexLevel* pairs, const float* mips, const float* trs, int sms, cudaStream_t s) {
    PairTable t{};
    for (int L = 1; L < kGtexPairs; ++L) {
        if (!pairs[L].surf || pairs[L].n != (256 >> L)) return cudaErrorInvalidValue;
        t.mip[L] = mips + mip_offset(L);
        t.tr[L] = trs + tr_offset(L - 1);
        t.surf[L] = pairs[L].surf;
        t.n[L] = pairs[L].n;
    }
    const size_t most = (size_t)130 * 130 * 130;
    const size_t want = (most + 255) / 256;
    const unsigned bx = (unsigned)(want < (size_t)sms * 8 ? want : (size_t)sms * 8);
    k_fill_pairs<<<dim3(bx, kGtexPairs), 256, 0, s>>>(t);   // row 0 (n = 0) returns at once
    return cudaGetLastError();
}

size_t gtex_pair_bytes(int n) { return (size_t)(n + 2) * (n + 2) * (n + 2) * sizeof(__half2); }

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
