// ref_prelude.h -- host stand-ins for the CUDA language features the
// reference's render sources use, so that those sources (compiled where they
// lie, unmodified) build as plain C++ for the CPU checker in oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY.  Force-included (-include) before every reference
// translation unit by oracle/Makefile.
#pragma once
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <barrier>
#include <thread>
#include <type_traits>
#include <vector>

#define __device__
#define __host__
#define __global__
#define __constant__
#define __forceinline__ inline
#define __restrict__ __restrict

#include "vector_types.h"

// CUDA device code resolves pow(float, float), exp(float), ... to the float
// overloads; bring std's overloads into the global namespace (one by one:
// C++20's std::lerp would clash with the reference's own lerp).
using std::abs; using std::acos; using std::atan; using std::atan2; using std::ceil; using std::cos;
using std::exp; using std::fabs; using std::floor; using std::fmax; using std::fmin; using std::log;
using std::pow; using std::sin; using std::sqrt; using std::tan;

// CUDA's host/device min/max overloads for scalars.
inline float max(float a, float b) { return fmaxf(a, b); }
inline float min(float a, float b) { return fminf(a, b); }
inline double max(double a, double b) { return fmax(a, b); }
inline double min(double a, double b) { return fmin(a, b); }
inline int max(int a, int b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
inline unsigned max(unsigned a, unsigned b) { return a > b ? a : b; }
inline unsigned min(unsigned a, unsigned b) { return a < b ? a : b; }
inline float saturate(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// Thread / block indices read by InitRand (values do not matter: the shim's
// curand_init takes its stream from the harness, see below).
extern thread_local uint3 threadIdx, blockIdx;
extern thread_local dim3 blockDim, gridDim;

// The reference reads the lane id with inline PTX,
//   asm volatile ("mov.u32 %0, %laneid;" : "=r"(ret));   (core/radiancePredict.cuh:8-12)
// This function-like macro (defined after every standard header above, so no
// library code sees it) turns that statement into an empty GNU asm whose
// output is tied to the emulated lane id of the calling host thread.
unsigned ref_shim_lane();
#define volatile(...) ("" : "=r"(ret) : "0"(ref_shim_lane()))

// Warp intrinsics, emulated by running the 32 lanes of a warp as 32 host
// threads that meet at a barrier for every collective (ref_harness.cpp).
float __shfl_sync(unsigned mask, float var, int src_lane, int width = 32);
unsigned __ballot_sync(unsigned mask, int predicate);
void __syncwarp(unsigned mask = 0xffffffffu);

// curand stand-in.  The reference seeds curand XORWOW per thread
// (core/render.cuh:49-58); the checker instead draws the build's
// Philox-4x32-10 stream selected by the harness, so both sides see the same
// random numbers.
struct curandState {
    uint32_t key[2];
    uint32_t sub, frame, kind, n;
};
void curand_init(unsigned long long seed, unsigned long long subsequence, unsigned long long offset,
                 curandState* state);
float curand_uniform(curandState* state);

// Texture-reference stand-in: a bound host array sampled in software with
// normalized coordinates and linear filtering.
#define cudaTextureType1D 0x01
#define cudaTextureType2D 0x02
#define cudaTextureType3D 0x03
enum cudaTextureReadMode { cudaReadModeElementType = 0, cudaReadModeNormalizedFloat = 1 };
enum cudaTextureFilterMode { cudaFilterModePoint = 0, cudaFilterModeLinear = 1 };
enum cudaTextureAddressMode { cudaAddressModeWrap = 0, cudaAddressModeClamp = 1,
                              cudaAddressModeMirror = 2, cudaAddressModeBorder = 3 };

template <class T, int Dim = cudaTextureType1D, int Mode = cudaReadModeElementType>
struct texture {
    int normalized = 1;
    cudaTextureFilterMode filterMode = cudaFilterModeLinear;
    cudaTextureAddressMode addressMode[3] = {cudaAddressModeBorder, cudaAddressModeBorder,
                                             cudaAddressModeBorder};
    const T* data = nullptr;
    int nx = 0, ny = 0, nz = 0;
    T constant{};   // returned by 2D float4 fetches (constant environment)
};

float ref_shim_lerp(float a, float b, float v);
float ref_shim_fetch3(const float* d, int nx, int ny, int nz, int x, int y, int z, bool clamp);

template <class T, int D, int M>
T tex3D(const texture<T, D, M>& t, float x, float y, float z) {
    if (!t.data) return T{};
    float px = x * (float)t.nx - 0.5f, py = y * (float)t.ny - 0.5f, pz = z * (float)t.nz - 0.5f;
    int ix = (int)floorf(px), iy = (int)floorf(py), iz = (int)floorf(pz);
    float wx = px - (float)ix, wy = py - (float)iy, wz = pz - (float)iz;
    bool cl = t.addressMode[0] == cudaAddressModeClamp;
    auto F = [&](int a, int b, int c) { return ref_shim_fetch3((const float*)t.data, t.nx, t.ny, t.nz, a, b, c, cl); };
    // fastest axis (texture x) innermost, as the oracle's software sampler
    float c00 = ref_shim_lerp(F(ix, iy, iz), F(ix + 1, iy, iz), wx);
    float c01 = ref_shim_lerp(F(ix, iy + 1, iz), F(ix + 1, iy + 1, iz), wx);
    float c10 = ref_shim_lerp(F(ix, iy, iz + 1), F(ix + 1, iy, iz + 1), wx);
    float c11 = ref_shim_lerp(F(ix, iy + 1, iz + 1), F(ix + 1, iy + 1, iz + 1), wx);
    return ref_shim_lerp(ref_shim_lerp(c00, c01, wy), ref_shim_lerp(c10, c11, wy), wz);
}

template <class T, int D, int M>
T tex2D(const texture<T, D, M>& t, float x, float y) {
    if constexpr (std::is_same<T, float>::value) {
        if (!t.data) return 0.0f;
        float px = x * (float)t.nx - 0.5f, py = y * (float)t.ny - 0.5f;
        int ix = (int)floorf(px), iy = (int)floorf(py);
        float wx = px - (float)ix, wy = py - (float)iy;
        auto F = [&](int a, int b) {
            a = a < 0 ? 0 : (a > t.nx - 1 ? t.nx - 1 : a);
            b = b < 0 ? 0 : (b > t.ny - 1 ? t.ny - 1 : b);
            return t.data[(size_t)b * t.nx + a];
        };
        // row (v) first, then u -- the order the oracle and kernels use
        float r0 = ref_shim_lerp(F(ix, iy), F(ix, iy + 1), wy);
        float r1 = ref_shim_lerp(F(ix + 1, iy), F(ix + 1, iy + 1), wy);
        return ref_shim_lerp(r0, r1, wx);
    } else if constexpr (std::is_same<T, float4>::value) {
        // environment map: wrap addressing, bilinear in software with fp32
        // weights, u (x) interpolated first -- the order of the reference's
        // own CPU sampler Image_host::Sample (core/volume.hpp:35-42); with no
        // map bound, the constant environment
        if (!t.data) return t.constant;
        float px = x * (float)t.nx - 0.5f, py = y * (float)t.ny - 0.5f;
        int ix = (int)floorf(px), iy = (int)floorf(py);
        float wx = px - (float)ix, wy = py - (float)iy;
        auto W = [](int a, int n) { a %= n; return a < 0 ? a + n : a; };
        auto F = [&](int a, int b) { return t.data[(size_t)W(b, t.ny) * t.nx + W(a, t.nx)]; };
        auto L = [&](float4 a, float4 b, float w) {
            return float4{ref_shim_lerp(a.x, b.x, w), ref_shim_lerp(a.y, b.y, w), ref_shim_lerp(a.z, b.z, w),
                          ref_shim_lerp(a.w, b.w, w)};
        };
        return L(L(F(ix, iy), F(ix + 1, iy), wx), L(F(ix, iy + 1), F(ix + 1, iy + 1), wx), wy);
    } else {
        return t.constant;
    }
}
