// mlp_tc.cu -- the MRPNN network (RadiancePredictInternal,
// core/radiancePredict.cu:301-422) on the 5th-generation tensor cores.
//
// Layout of the work.  A persistent kernel with one CTA per SM holds every
// layer's weights in shared memory as UMMA operand images (K-major, no
// swizzle: 8-row x 16-byte core matrices).  Two groups of 128 threads each
// own one 128-pixel tile at a time; thread t of a group owns pixel row t of
// its tile and TMEM lane t.  Per layer step the group writes its A rows
// (activations, rounded to BF16 or quantised to FP8-E4M3) to shared memory,
// one elected thread issues tcgen05.mma into the group's TMEM columns and
// commits to an mbarrier, and every thread reads its row of the FP32
// accumulator back with tcgen05.ld for the epilogue (bias, ReLU, residuals,
// gates), all in FP32 on the CUDA cores.  The SE gate MLPs, pooling, the
// LSEFin gate and the last 16->1 layer stay in FP32.
//
// Layers (58): per SE block three branch layers w x w (main widths 8, 8, 16,
// 16, 16, 32, 32, 32; direct-illumination 4 x 8), the three final 32x32 and
// 8x8 layers, then LC0 128x128, LC1 64x128, LC2 32x64, LX 16x32, LX0..LX11
// 16x16.  N and K are padded to the MMA granularity with zeros.
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_fp16.h>

#include "kernels.h"
#include "mlp_tc.h"
#include "tc_ptx.cuh"

namespace mrp {

// ---------------------------------------------------------------------------
// layer table (shared by the host packer and the kernel)
// ---------------------------------------------------------------------------
constexpr int kLayers = 58;
// main SE block widths (kMainW) and packed fp32 offsets, usable at run time in device code
__host__ __device__ constexpr int mw(int k) { return k < 2 ? 8 : k < 5 ? 16 : 32; }
__host__ __device__ constexpr int mblk_off(int k) { int o = 0; for (int i = 0; i < k; ++i) o += 64 + 24 + 3 * (mw(i) * mw(i) + mw(i)); return o; }
static_assert(mblk_off(8) == kMainFinalOff, "block offsets");
constexpr int kL81 = 24, kLD41 = 39, kLC0 = 42, kLC1 = 43, kLC2 = 44, kLX = 45, kLX0 = 46;
__host__ __device__ constexpr int layer_n(int i) {
    return i < 24 ? mw(i / 3) : i < 27 ? 32 : i < 42 ? 8 : i == kLC0 ? 128 : i == kLC1 ? 64 : i == kLC2 ? 32 : 16;
}
__host__ __device__ constexpr int layer_k(int i) {
    return i < 24 ? mw(i / 3) : i < 27 ? 32 : i < 42 ? 8 : i == kLC0 ? 128 : i == kLC1 ? 128 : i == kLC2 ? 64 :
           i == kLX ? 32 : 16;
}
__host__ __device__ constexpr int pad_to(int x, int m) { return (x + m - 1) / m * m; }
// operand element bytes: 2 (BF16) or 1 (E4M3); K granularity 16 / 32 elements
__host__ __device__ constexpr int kpad(int i, int eb) { return pad_to(layer_k(i), eb == 2 ? 16 : 32); }
__host__ __device__ constexpr int npad(int i) { return pad_to(layer_n(i), 16); }
__host__ __device__ constexpr int layer_bytes(int i, int eb) { return npad(i) * kpad(i, eb) * eb; }
__host__ __device__ constexpr int layer_off(int i, int eb) {
    int o = 0;
    for (int j = 0; j < i; ++j) o += layer_bytes(j, eb);
    return o;
}
__host__ __device__ constexpr int image_bytes(int eb) { return layer_off(kLayers, eb); }
// FP8 weight scales: one per output channel, layer i's at scale_off(i)
__host__ __device__ constexpr int scale_off(int i) {
    int o = 0;
    for (int j = 0; j < i; ++j) o += npad(j);
    return o;
}
constexpr int kScaleCount = scale_off(kLayers);
// The fp32 constants the CUDA-core parts read, packed for shared memory:
// FP8 weight scales, layer biases (both indexed by scale_off), the 12 SE gate
// MLPs (8x8 + 3x8 each), LSEFin1 / LSEFin2, LGGS and the 16 -> 1 head.
constexpr int kAuxScale = 0, kAuxBias = kScaleCount, kAuxSE = 2 * kScaleCount, kAuxLSE1 = kAuxSE + 12 * 88,
              kAuxLSE2 = kAuxLSE1 + 1200, kAuxLGGSW = kAuxLSE2 + 96, kAuxLGGSB = kAuxLGGSW + 24,
              kAuxLX12W = kAuxLGGSB + 8, kAuxLX12B = kAuxLX12W + 16, kAuxCount = (kAuxLX12B + 1 + 3) / 4 * 4;
// fp32 weight / bias of layer i in the packed fp32 layout (common.cuh)
__host__ __device__ constexpr int layer_w32(int i) {
    return i < 24 ? mblk_off(i / 3) + 88 + (i % 3) * (mw(i / 3) * mw(i / 3) + mw(i / 3))
         : i < 27 ? kMainFinalOff + (i - 24) * (1024 + 32)
         : i < 39 ? di_block_off((i - 27) / 3) + 88 + ((i - 27) % 3) * 72
         : i < 42 ? kDiFinalOff + (i - 39) * 72
         : i == kLC0 ? kLC0W : i == kLC1 ? kLC1W : i == kLC2 ? kLC2W : i == kLX ? kLXW : lxw(i - kLX0);
}
__host__ __device__ constexpr int layer_b32(int i) { return layer_w32(i) + layer_n(i) * layer_k(i); }
static_assert(layer_b32(kLC0) == kLC0B && layer_b32(kLX0 + 11) == lxb(11), "layer table");
static_assert(image_bytes(2) <= 110 * 1024, "BF16 weight image must fit shared memory");
static_assert(kAuxBias % 4 == 0 && kAuxSE % 4 == 0 && kAuxLSE1 % 4 == 0 && kAuxLSE2 % 4 == 0 && 88 % 4 == 0,
              "constants read as float4 start on 16-byte boundaries");

// Byte offset of element (row m, k) in a K-major no-swizzle operand tile of
// padded width Kp: 8-row groups SBO = Kp*eb*8 bytes apart, 16-byte K chunks
// 128 bytes apart, rows of a core matrix 16 bytes apart.
__host__ __device__ constexpr int op_off(int m, int k, int kp, int eb) {
    return (m / 8) * (kp * eb * 8) + (k * eb / 16) * 128 + (m % 8) * 16 + (k * eb) % 16;
}

// ---------------------------------------------------------------------------
// host: operand images
// ---------------------------------------------------------------------------
static uint16_t bf16_bits(float f) {   // round to nearest even
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16 | ((u & 0xFFFF) ? 0x40 : 0));
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
// E4M3 (bias 7, no infinities, max 448), round to nearest even, saturating.
static uint8_t e4m3_bits(float f) {
    uint8_t s = std::signbit(f) ? 0x80 : 0;
    double a = std::fabs((double)f);
    if (!(a == a)) return 0x7F;
    if (a >= 448.0) return s | 0x7E;
    if (a < std::ldexp(1.0, -10)) return s;   // below half the smallest subnormal
    int e;
    std::frexp(a, &e);                        // a = m * 2^e, m in [0.5, 1)
    int ex = e - 1;                           // a in [2^ex, 2^(ex+1))
    if (ex < -6) ex = -6;                     // subnormal range shares 2^-6 * 0.mmm
    double q = std::ldexp(1.0, ex - 3);       // quantum of 3 mantissa bits
    double n = std::nearbyint(a / q);         // ties to even (default rounding)
    double v = n * q;
    if (v >= 448.0) return s | 0x7E;
    if (v == 0) return s;
    int vex;
    std::frexp(v, &vex);
    vex -= 1;
    if (vex < -6) return s | (uint8_t)(v / std::ldexp(1.0, -9));   // subnormal: mantissa / 8 * 2^-6
    uint8_t mant = (uint8_t)(v / std::ldexp(1.0, vex) * 8.0 - 8.0);
    return s | (uint8_t)((vex + 7) << 3) | mant;
}

static cudaError_t upload_layer_descs();
cudaError_t tc_prepare_weights(const float* w32, TcWeights& w) {
    std::vector<uint8_t> img16(image_bytes(2), 0), img8(image_bytes(1), 0);
    // FP8: each output channel (weight row) scaled by its own amax / 448
    std::vector<float> scales(kScaleCount, 1.0f);
    for (int i = 0; i < kLayers; ++i) {
        int n = layer_n(i), k = layer_k(i);
        const float* W = w32 + layer_w32(i);   // [n][k], row-major (Out, In)
        for (int r = 0; r < n; ++r) {
            float amax = 0.0f;
            for (int c = 0; c < k; ++c) amax = std::fmax(amax, std::fabs(W[r * k + c]));
            float s = amax > 0 ? amax / 448.0f : 1.0f;
            scales[scale_off(i) + r] = s;
            for (int c = 0; c < k; ++c) {
                uint16_t b = bf16_bits(W[r * k + c]);
                std::memcpy(&img16[layer_off(i, 2) + op_off(r, c, kpad(i, 2), 2)], &b, 2);
                img8[layer_off(i, 1) + op_off(r, c, kpad(i, 1), 1)] = e4m3_bits(W[r * k + c] / s);
            }
        }
    }
    std::vector<float> aux(kAuxCount, 0.0f);
    for (int i = 0; i < kScaleCount; ++i) aux[kAuxScale + i] = scales[i];
    for (int i = 0; i < kLayers; ++i)
        for (int r = 0; r < layer_n(i); ++r) aux[kAuxBias + scale_off(i) + r] = w32[layer_b32(i) + r];
    for (int b = 0; b < 12; ++b) {
        const float* src = w32 + (b < 8 ? mblk_off(b) : di_block_off(b - 8));
        std::memcpy(&aux[kAuxSE + 88 * b], src, 88 * sizeof(float));
    }
    // LSEFin1 [16][75] (out, in) stored input-major [75][16]
    for (int o = 0; o < 16; ++o)
        for (int j = 0; j < 75; ++j) aux[kAuxLSE1 + 16 * j + o] = w32[kLSEFin1W + o * 75 + j];
    std::memcpy(&aux[kAuxLSE2], w32 + kLSEFin2W, 96 * sizeof(float));
    std::memcpy(&aux[kAuxLGGSW], w32 + kLGGSW, 24 * sizeof(float));
    std::memcpy(&aux[kAuxLGGSB], w32 + kLGGSB, 8 * sizeof(float));
    std::memcpy(&aux[kAuxLX12W], w32 + kLX12W, 16 * sizeof(float));
    aux[kAuxLX12B] = w32[kLX12B];
    cudaError_t e;
    if (!w.d_aux && (e = mrp::dev_malloc(&w.d_aux, kAuxCount * sizeof(float))) != cudaSuccess) return e;
    if ((e = cudaMemcpy(w.d_aux, aux.data(), kAuxCount * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
        return e;
    if (!w.d_bf16 && (e = mrp::dev_malloc(&w.d_bf16, img16.size())) != cudaSuccess) return e;
    if (!w.d_fp8 && (e = mrp::dev_malloc(&w.d_fp8, img8.size())) != cudaSuccess) return e;
    if (!w.d_scales && (e = mrp::dev_malloc(&w.d_scales, kScaleCount * sizeof(float))) != cudaSuccess) return e;
    if (!w.d_err && (e = mrp::dev_malloc(&w.d_err, sizeof(int))) != cudaSuccess) return e;
    if (!w.d_counter && (e = mrp::dev_malloc(&w.d_counter, sizeof(int))) != cudaSuccess) return e;
    if ((e = cudaMemcpy(w.d_bf16, img16.data(), img16.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(w.d_fp8, img8.data(), img8.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(w.d_scales, scales.data(), kScaleCount * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
        return e;
    if ((e = cudaMemset(w.d_err, 0, sizeof(int))) != cudaSuccess) return e;
    if ((e = upload_layer_descs()) != cudaSuccess) return e;
    w.ready = true;
    return cudaSuccess;
}
cudaError_t tc_ensure_scratch(TcScratch& s) {
    if (s.d) return cudaSuccess;
    cudaError_t e = mrp::dev_malloc(&s.d, 2 * sizeof(int));
    if (e != cudaSuccess) { s.d = nullptr; return e; }
    return cudaMemset(s.d, 0, 2 * sizeof(int));
}
void tc_free_scratch(TcScratch& s) {
    if (s.d) mrp::dev_free(s.d);
    s.d = nullptr;
}

// ---------------------------------------------------------------------------
// device: layer descriptors, group synchronisation, one MMA round
//
// Code size matters here: the whole network runs inside one kernel and two
// groups execute different layers at once, so every layer of one shape
// shares one routine and takes its layer index at run time from a constant
// table (instead of one template instance per layer).
// ---------------------------------------------------------------------------
constexpr int kGroupThreads = 128;
constexpr int kGroups = 2;
constexpr int kTmemColsPerGroup = 256;
constexpr uint32_t kWaitLimit = 1u << 22;   // polls before an MMA round is declared lost
constexpr int kABytes = 128 * 128 * 2;      // one group's A buffer (largest: 128 x 128 BF16)

struct LayerDesc {
    int b_off[2];   // byte offset of the weight image, [0] BF16, [1] E4M3
    int kp[2];      // padded K
    int n, np;      // logical / padded N
    int abias;      // bias offset in the shared-memory constants (kAuxBias + scale_off)
    int soff;       // FP8 scale offset
};
__constant__ LayerDesc c_layer_desc[kLayers];

static void fill_layer_descs(LayerDesc* d) {
    for (int i = 0; i < kLayers; ++i) {
        d[i].b_off[0] = layer_off(i, 2);
        d[i].b_off[1] = layer_off(i, 1);
        d[i].kp[0] = kpad(i, 2);
        d[i].kp[1] = kpad(i, 1);
        d[i].n = layer_n(i);
        d[i].np = npad(i);
        d[i].abias = kAuxBias + scale_off(i);
        d[i].soff = scale_off(i);
    }
}

static cudaError_t upload_layer_descs() {
    LayerDesc descs[kLayers];
    fill_layer_descs(descs);
    return cudaMemcpyToSymbol(c_layer_desc, descs, sizeof descs);
}

__device__ __forceinline__ void group_bar(int g) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(kGroupThreads) : "memory");
}

// Per-thread constants of a group, passed by value into the per-block
// routines (a reference would put them in local memory and make every use a
// load).  The mutable part -- mbarrier phase (bit 0) and "a wait timed out"
// (bit 1) -- travels as an int through the calls.
struct Group {
    int g, t;             // group index, thread within the group
    uint32_t a_s;         // A buffer (shared address)
    uint32_t wimg_s;      // weight image (shared address)
    uint32_t mbar_s;      // the group's mbarrier (shared address)
    uint32_t tmem;        // TMEM address of this thread's lane, column 0 of the group
    int* err;
};
constexpr int kStFailed = 2;

// Up to three MMAs (layer, A sub-tile byte offset, D column), issued after
// all A rows are in shared memory and awaited by the whole group.
template <int EB>
__device__ __noinline__ int mma_round(const Group G, int st, int count, int l0, int a_stride, int d0, int d_stride) {
    tc::fence_proxy_async();
    tc::fence_before_sync();
    group_bar(G.g);
    if (G.t == 0) {
        tc::fence_after_sync();
        const uint32_t col0 = G.tmem & 0xFFFFu;   // lane 0, the group's column 0
        const int e = EB == 2 ? 0 : 1;
#pragma unroll 1
        for (int q = 0; q < count; ++q) {
            const int L = l0 + q;
            int kp = c_layer_desc[L].kp[e];
            uint32_t idesc = tc::instr_desc(128, c_layer_desc[L].np, EB == 2 ? tc::kFmtBF16 : tc::kFmtE4M3);
            uint32_t sbo = (uint32_t)(kp * EB * 8);
            int steps = kp * EB / 32;   // 32 bytes of K per MMA (16 BF16 / 32 E4M3)
            uint32_t ab = G.a_s + (uint32_t)(q * a_stride), bb = G.wimg_s + (uint32_t)c_layer_desc[L].b_off[e];
            uint32_t dc = col0 + (uint32_t)(d0 + q * d_stride);
#pragma unroll 1
            for (int s = 0; s < steps; ++s) {
                uint64_t ad = tc::smem_desc(ab + s * 256, 128, sbo);
                uint64_t bd = tc::smem_desc(bb + s * 256, 128, sbo);
                if (EB == 2) tc::mma_bf16(dc, ad, bd, idesc, s > 0);
                else tc::mma_fp8(dc, ad, bd, idesc, s > 0);
            }
        }
        tc::mma_commit_s(G.mbar_s);
    }
    bool done = tc::mbar_wait_s(G.mbar_s, (uint32_t)(st & 1), kWaitLimit);
    st ^= 1;
    if (!done) {
        st |= kStFailed;
        atomicExch(G.err, 1);
    }
    tc::fence_after_sync();
    return st;
}

// Writes this thread's row of an A operand: v[0..n) (zero padded to kp) at
// sub-tile byte offset `off`.  FP8 rows are scaled by 1/s (s = row amax/448),
// returned so the epilogue can undo it.
template <int EB, int N, int KP>
__device__ __forceinline__ float write_row(uint32_t a_s, int off, int row, const float* v) {
    float inv = 1.0f, s = 1.0f;
    if (EB == 1) {
        float amax = 0.0f;
#pragma unroll
        for (int i = 0; i < N; ++i) amax = fmaxf(amax, fabsf(v[i]));
        s = amax > 0.0f ? amax * (1.0f / 448.0f) : 1.0f;
        inv = 1.0f / s;
    }
    constexpr int E = 16 / EB;   // elements per 16-byte chunk
#pragma unroll
    for (int c = 0; c < KP / E; ++c) {
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (EB == 2) {
                int i0 = c * 8 + 2 * q;
                float lo = i0 < N ? v[i0] : 0.0f, hi = i0 + 1 < N ? v[i0 + 1] : 0.0f;
                w[q] = tc::pack_bf16(lo, hi);
            } else {
                int i0 = c * 16 + 4 * q;
                float x0 = i0 < N ? v[i0] * inv : 0.0f, x1 = i0 + 1 < N ? v[i0 + 1] * inv : 0.0f;
                float x2 = i0 + 2 < N ? v[i0 + 2] * inv : 0.0f, x3 = i0 + 3 < N ? v[i0 + 3] * inv : 0.0f;
                w[q] = (uint32_t)tc::pack_e4m3(x0, x1) | ((uint32_t)tc::pack_e4m3(x2, x3) << 16);
            }
        }
        tc::st_shared_v4(a_s + (uint32_t)(off + op_off(row, c * E, KP, EB)), w[0], w[1], w[2], w[3]);
    }
    return s;
}

// Reads N (<= 128) accumulator columns of this thread's row.
template <int N>
__device__ __forceinline__ void read_cols(const Group& G, int col, float* out) {
#pragma unroll
    for (int c = 0; c < (N + 15) / 16; ++c) {
        float v[16];
        tc::tmem_ld16(G.tmem + col + 16 * c, v);
#pragma unroll
        for (int i = 0; i < 16; ++i)
            if (16 * c + i < N) out[16 * c + i] = v[i];
    }
}

MRP_D float wl(const float* __restrict__ w, int i) { return __ldg(w + i); }
MRP_D float sigmoid_d(float o) { return 1.0f / (1.0f + __expf(-o)); }

// relu(D * scale + b) for N columns of layer L (runtime), in place.
// The constants live in shared memory but reach the routines as a generic
// pointer; reading them with shared-space loads (the address converted once
// per access) keeps them off the generic load path, whose results the
// scheduler tracks like global loads.
MRP_D float4 lds4(const float* p) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}
MRP_D float lds1(const float* p) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}

// Biases and scales start on 16-float boundaries (scale_off), so they are
// read four at a time.
template <int EB, int N>
MRP_D void bias_relu(float* d, int L, float rs, const float* aux) {
    static_assert(N % 4 == 0, "layer widths are multiples of 4");
    const int ab = c_layer_desc[L].abias, so = c_layer_desc[L].soff;
#pragma unroll
    for (int q = 0; q < N / 4; ++q) {
        const float4 b = lds4(aux + ab + 4 * q);
        float4 sc = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        if (EB == 1) {
            const float4 w = lds4(aux + kAuxScale + so + 4 * q);
            sc = make_float4(rs * w.x, rs * w.y, rs * w.z, rs * w.w);
        }
        d[4 * q] = fmaxf(fmaf(d[4 * q], sc.x, b.x), 0.0f);
        d[4 * q + 1] = fmaxf(fmaf(d[4 * q + 1], sc.y, b.y), 0.0f);
        d[4 * q + 2] = fmaxf(fmaf(d[4 * q + 2], sc.z, b.z), 0.0f);
        d[4 * q + 3] = fmaxf(fmaf(d[4 * q + 3], sc.w, b.w), 0.0f);
    }
}
// n consecutive constants (16-byte aligned, n a multiple of 4) into registers.
template <int N>
MRP_D void aux_row(const float* aux, int off, float* out) {
#pragma unroll
    for (int q = 0; q < N / 4; ++q) {
        const float4 v = lds4(aux + off + 4 * q);
        out[4 * q] = v.x; out[4 * q + 1] = v.y; out[4 * q + 2] = v.z; out[4 * q + 3] = v.w;
    }
}

// Feature sources (rows may be invalid: zeros); FROM is a run-time offset.
struct RowFeatures {           // [n][576] row-major
    const float* x;
    bool valid;
    template <int W>
    MRP_D void load(int c, int from, float* xs) const {
#pragma unroll
        for (int i = 0; i < W; ++i) xs[i] = valid ? __ldg(x + c * 192 + from + i) : 0.0f;
    }
};
struct TileFeatures {          // FP16 pairs of the staged predictor's tiled layout
    const __half2* x;          // already offset to (r / 32) * 288 * 32 + r % 32
    bool valid;
    template <int W>
    MRP_D void load(int c, int from, float* xs) const {
#pragma unroll
        for (int k = 0; k < W / 2; ++k) {
            const float2 p = valid ? __half22float2(__ldg(x + (c * 96 + (from >> 1) + k) * 32)) : make_float2(0.0f, 0.0f);
            xs[2 * k] = p.x;
            xs[2 * k + 1] = p.y;
        }
    }
};

// Per-row state that lives in TMEM between blocks (columns of the group's
// 256; the MMA accumulators use 0..95 (main blocks, finals), 128..175 (DI
// blocks), 176..223 (DI finals)): the LSEFin1 partial sums and the residual
// of the main (3 x 32) and direct-illumination (3 x 8) chains.  Keeping them
// out of registers leaves the per-block routines without a stack frame for
// them.
constexpr int kColHf = 96, kColPrevMain = 160, kColPrevDi = 232;

template <int N>
MRP_D void tmem_get(const Group& G, int col, float* out) {
    if constexpr (N == 8) {
        uint32_t r[8];
        tc::tmem_ld8_nowait(G.tmem + col, r);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; ++i) out[i] = __uint_as_float(r[i]);
    } else {
        uint32_t r[N / 16][16];
#pragma unroll
        for (int c = 0; c < N / 16; ++c) tc::tmem_ld16_nowait(G.tmem + col + 16 * c, r[c]);
        tc::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < N / 16; ++c)
#pragma unroll
            for (int i = 0; i < 16; ++i) out[16 * c + i] = __uint_as_float(r[c][i]);
    }
}
template <int N>
MRP_D void tmem_put(const Group& G, int col, const float* v) {
    if constexpr (N == 8) {
        float t[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) t[i] = v[i];
        tc::tmem_st8(G.tmem + col, t);
    } else {
#pragma unroll
        for (int c = 0; c < N / 16; ++c) {
            float t[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) t[i] = v[16 * c + i];
            tc::tmem_st16(G.tmem + col + 16 * c, t);
        }
    }
}

struct BlockDesc { int w, from, widen, has_prev, l0, dcol, se_off, pid, pcol, pstride; };
__constant__ BlockDesc c_blocks[12] = {
    {8, 0, 0, 0, 0, 0, kAuxSE + 88 * 0, 0, kColPrevMain, 32},      {8, 8, 1, 1, 3, 0, kAuxSE + 88 * 1, 3, kColPrevMain, 32},
    {16, 16, 0, 1, 6, 0, kAuxSE + 88 * 2, 6, kColPrevMain, 32},    {16, 32, 0, 1, 9, 0, kAuxSE + 88 * 3, 9, kColPrevMain, 32},
    {16, 48, 1, 1, 12, 0, kAuxSE + 88 * 4, 12, kColPrevMain, 32},  {32, 64, 0, 1, 15, 0, kAuxSE + 88 * 5, 15, kColPrevMain, 32},
    {32, 96, 0, 1, 18, 0, kAuxSE + 88 * 6, 18, kColPrevMain, 32},  {32, 128, 0, 1, 21, 0, kAuxSE + 88 * 7, 21, kColPrevMain, 32},
    {8, 160, 0, 0, 27, 128, kAuxSE + 88 * 8, 24, kColPrevDi, 8}, {8, 168, 0, 1, 30, 128, kAuxSE + 88 * 9, 27, kColPrevDi, 8},
    {8, 176, 0, 1, 33, 128, kAuxSE + 88 * 10, 30, kColPrevDi, 8}, {8, 184, 0, 1, 36, 128, kAuxSE + 88 * 11, 33, kColPrevDi, 8},
};

// One SE block over the three channels (SE / SERES + ADD3 / REP3,
// core/radiancePredict.cu:240-294): gate from the slice pools, branch layers
// l0..l0+2 on the tensor cores (D at dcol, dcol+stride, dcol+2*stride), then
// prev <- relu(D + b) + slice (ADD3) or concat(relu(D + b), slice) (REP3).
template <int EB, int W, class Src>
__device__ __noinline__ int tc_block(const Group G, int st, const Src src, const float* aux, int b, float g,
                                     float gamma) {
    const BlockDesc bd = c_blocks[b];
    const int from = bd.from, widen = bd.widen, has_prev = bd.has_prev, l0 = bd.l0, dcol = bd.dcol,
              se_off = bd.se_off, pid = bd.pid, pcol = bd.pcol, pstride = bd.pstride;
    constexpr int KP = pad_to(W, EB == 2 ? 16 : 32);
    constexpr int SUB = 128 * KP * EB;   // bytes of one branch's A sub-tile
    constexpr int DSTR = W <= 16 ? 16 : 32;
    float xs[3][W];                      // the block's feature slice, loaded once
    float p8[8];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        src.template load<W>(c, from, xs[c]);
        float s = 0.0f, m = -10000.0f;
#pragma unroll
        for (int i = 0; i < W; ++i) { s += xs[c][i]; m = fmaxf(m, xs[c][i]); }
        p8[c] = s / (float)W;
        p8[3 + c] = m;
    }
    p8[6] = g;
    p8[7] = gamma;
    // LSEFin1 (75 -> 16) accumulated block by block in TMEM: pool[pid + c] =
    // avg, pool[36 + pid + c] = max
    {
        float hf[16];
        tmem_get<16>(G, kColHf, hf);
        // (LSEFin1 is stored input-major: the 16 weights of input j at
        // kAuxLSE1 + 16 j; per output the same sequence of FMAs as o-major)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float wa[16], wm[16];
            aux_row<16>(aux, kAuxLSE1 + 16 * (pid + c), wa);
            aux_row<16>(aux, kAuxLSE1 + 16 * (36 + pid + c), wm);
#pragma unroll
            for (int o = 0; o < 16; ++o) {
                hf[o] = fmaf(wa[o], p8[c], hf[o]);
                hf[o] = fmaf(wm[o], p8[3 + c], hf[o]);
            }
        }
        tmem_put<16>(G, kColHf, hf);
    }
    float h[8], gate[3];
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        float w[8];
        aux_row<8>(aux, se_off + o * 8, w);
        float a = 0.0f;
#pragma unroll
        for (int j = 0; j < 8; ++j) a = fmaf(p8[j], w[j], a);
        h[o] = fmaxf(a, 0.0f);
    }
#pragma unroll
    for (int o = 0; o < 3; ++o) {
        float w[8];
        aux_row<8>(aux, se_off + 64 + o * 8, w);
        float a = 0.0f;
#pragma unroll
        for (int j = 0; j < 8; ++j) a = fmaf(h[j], w[j], a);
        gate[o] = sigmoid_d(a);
    }
    float rs[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float in[W];
        if (has_prev) {
            float pv[W];
            tmem_get<W>(G, pcol + c * pstride, pv);
#pragma unroll
            for (int i = 0; i < W; ++i) in[i] = fmaf(xs[c][i], gate[c], pv[i]);
        } else {
#pragma unroll
            for (int i = 0; i < W; ++i) in[i] = xs[c][i] * gate[c];
        }
        rs[c] = write_row<EB, W, KP>(G.a_s, c * SUB, G.t, in);
    }
    st = mma_round<EB>(G, st, 3, l0, SUB, dcol, DSTR);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float d[W];
        read_cols<W>(G, dcol + c * DSTR, d);
        bias_relu<EB, W>(d, l0 + c, rs[c], aux);
        if (widen) {
            float nv[2 * W];
#pragma unroll
            for (int o = 0; o < W; ++o) { nv[o] = d[o]; nv[W + o] = xs[c][o]; }
            tmem_put<2 * W>(G, pcol + c * pstride, nv);
        } else {
#pragma unroll
            for (int o = 0; o < W; ++o) d[o] = d[o] + xs[c][o];
            tmem_put<W>(G, pcol + c * pstride, d);
        }
    }
    tc::tmem_wait_st();
    return st;
}

// Residual pair k of the tail: a += relu(LX(2k+1) relu(LX(2k) a + b) + b),
// a (16 values) kept in TMEM columns kColA16.
constexpr int kColA16 = 96;
template <int EB>
__device__ __noinline__ int tc_residual_pair(const Group G, int st, const float* aux, int k) {
    constexpr int KP = EB == 2 ? 16 : 32;
    const int La = kLX0 + 2 * k, Lb = La + 1;
    float a16[16];
    tmem_get<16>(G, kColA16, a16);
    float r0 = write_row<EB, 16, KP>(G.a_s, 0, G.t, a16);
    st = mma_round<EB>(G, st, 1, La, 0, 64, 0);
    float u[16];
    read_cols<16>(G, 64, u);
    bias_relu<EB, 16>(u, La, r0, aux);
    float r1 = write_row<EB, 16, KP>(G.a_s, 0, G.t, u);
    st = mma_round<EB>(G, st, 1, Lb, 0, 80, 0);
    float z[16];
    read_cols<16>(G, 80, z);
    bias_relu<EB, 16>(z, Lb, r1, aux);
#pragma unroll
    for (int i = 0; i < 16; ++i) a16[i] += z[i];
    tmem_put<16>(G, kColA16, a16);
    tc::tmem_wait_st();
    return st;
}

// The tail of one albedo channel (core/radiancePredict.cu:375-419): LSEFin
// gate, LC0 over [comb * gate, LGGS], LC1, LC2, LX, six residual pairs and
// the 16 -> 1 head.  comb comes from TMEM (kColComb); the accumulators use
// columns 0..127 only, so comb survives for the next channel.
constexpr int kColComb = 136;
struct TailOut { float p; int st; };
// hf (the LSEFin1 partial sums) is read from TMEM columns kColHf first thing.
template <int EB>
__device__ __noinline__ TailOut tc_tail(const Group G, int st, const float* aux, float g, float gamma, float s4) {
    float h[16], gf[6];
    tmem_get<16>(G, kColHf, h);
#pragma unroll
    for (int o = 0; o < 16; ++o) {
        float a = h[o];
        a = fmaf(lds1(aux + kAuxLSE1 + 16 * 72 + o), g, a);
        a = fmaf(lds1(aux + kAuxLSE1 + 16 * 73 + o), gamma, a);
        a = fmaf(lds1(aux + kAuxLSE1 + 16 * 74 + o), s4, a);
        h[o] = fmaxf(a, 0.0f);
    }
#pragma unroll
    for (int o = 0; o < 6; ++o) {
        float w[16];
        aux_row<16>(aux, kAuxLSE2 + o * 16, w);
        float a = 0.0f;
#pragma unroll
        for (int j = 0; j < 16; ++j) a = fmaf(h[j], w[j], a);
        gf[o] = sigmoid_d(a);
    }
    // LC0's A row: [comb * gate segment, LGGS (3 -> 8)]
    float x[128];
    tmem_get<32>(G, kColComb, x);
    tmem_get<32>(G, kColComb + 32, x + 32);
    tmem_get<32>(G, kColComb + 64, x + 64);
    tmem_get<8>(G, kColComb + 96, x + 96);
    tmem_get<8>(G, kColComb + 104, x + 104);
    tmem_get<8>(G, kColComb + 112, x + 112);
#pragma unroll
    for (int i = 0; i < 120; ++i) x[i] = x[i] * gf[i < 96 ? i / 32 : 3 + (i - 96) / 8];
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        float a = 0.0f;
        a = fmaf(g, lds1(aux + kAuxLGGSW + o * 3), a);
        a = fmaf(gamma, lds1(aux + kAuxLGGSW + o * 3 + 1), a);
        a = fmaf(s4, lds1(aux + kAuxLGGSW + o * 3 + 2), a);
        x[120 + o] = fmaxf(a + lds1(aux + kAuxLGGSB + o), 0.0f);
    }
    float r = write_row<EB, 128, kpad(kLC0, EB)>(G.a_s, 0, G.t, x);
    st = mma_round<EB>(G, st, 1, kLC0, 0, 0, 0);
    read_cols<128>(G, 0, x);
    bias_relu<EB, 128>(x, kLC0, r, aux);
    r = write_row<EB, 128, kpad(kLC1, EB)>(G.a_s, 0, G.t, x);
    st = mma_round<EB>(G, st, 1, kLC1, 0, 0, 0);
    read_cols<64>(G, 0, x);
    bias_relu<EB, 64>(x, kLC1, r, aux);
    r = write_row<EB, 64, kpad(kLC2, EB)>(G.a_s, 0, G.t, x);
    st = mma_round<EB>(G, st, 1, kLC2, 0, 0, 0);
    read_cols<32>(G, 0, x);
    bias_relu<EB, 32>(x, kLC2, r, aux);
    r = write_row<EB, 32, kpad(kLX, EB)>(G.a_s, 0, G.t, x);
    st = mma_round<EB>(G, st, 1, kLX, 0, 32, 0);
    float a16[16];
    read_cols<16>(G, 32, a16);
    bias_relu<EB, 16>(a16, kLX, r, aux);
    tmem_put<16>(G, kColA16, a16);
    tc::tmem_wait_st();
#pragma unroll 1
    for (int k = 0; k < 6; ++k) st = tc_residual_pair<EB>(G, st, aux, k);
    tmem_get<16>(G, kColA16, a16);
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 16; ++j) a = fmaf(a16[j], lds1(aux + kAuxLX12W + j), a);
    return TailOut{fmaxf(a + lds1(aux + kAuxLX12B), 0.0f), st};
}


template <int EB, class Src>
MRP_D int run_block(const Group& G, int st, const Src& src, const float* aux, int b, float g, float gamma) {
    const int w = c_blocks[b].w;
    if (w == 8) return tc_block<EB, 8>(G, st, src, aux, b, g, gamma);
    if (w == 16) return tc_block<EB, 16>(G, st, src, aux, b, g, gamma);
    return tc_block<EB, 32>(G, st, src, aux, b, g, gamma);
}

template <int EB, class Src>
MRP_D int tc_network(const Group& G, int st, const Src& src, const float* aux,
                      float gamma, float g, f3 sr, float out[3]) {
    {
        float z[16];
#pragma unroll
        for (int o = 0; o < 16; ++o) z[o] = 0.0f;
        tmem_put<16>(G, kColHf, z);
        tc::tmem_wait_st();
    }
    // main branch, X[0:160]; the three 32x32 finals leave comb[0:96) in TMEM columns 0..95
#pragma unroll 1
    for (int b = 0; b < 8; ++b) st = run_block<EB>(G, st, src, aux, b, g, gamma);
    float rs_main[3];
    {
        constexpr int KP = pad_to(32, EB == 2 ? 16 : 32), SUB = 128 * KP * EB;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float pv[32];
            tmem_get<32>(G, kColPrevMain + 32 * c, pv);
            rs_main[c] = write_row<EB, 32, KP>(G.a_s, c * SUB, G.t, pv);
        }
        st = mma_round<EB>(G, st, 3, kL81, SUB, 0, 32);
    }
    // direct-illumination branch, X[160:192]; the 8x8 finals at columns 176..223
#pragma unroll 1
    for (int b = 8; b < 12; ++b) st = run_block<EB>(G, st, src, aux, b, g, gamma);
    float rs_di[3];
    {
        constexpr int KP = pad_to(8, EB == 2 ? 16 : 32), SUB = 128 * KP * EB;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float pv[8];
            tmem_get<8>(G, kColPrevDi + 8 * c, pv);
            rs_di[c] = write_row<EB, 8, KP>(G.a_s, c * SUB, G.t, pv);
        }
        st = mma_round<EB>(G, st, 3, kLD41, SUB, 176, 16);
    }
    float hf[16];
    tmem_get<16>(G, kColHf, hf);   // before LC0's accumulator covers columns 0..127
    // comb[120] = relu(finals + b) -> TMEM columns kColComb..+119: the DI
    // finals (176..223) first, then the main ones (0..95) -- the main comb
    // lands on 136..231, over DI columns already read.
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float e[8];
        read_cols<8>(G, 176 + 16 * c, e);
        bias_relu<EB, 8>(e, kLD41 + c, rs_di[c], aux);
        tmem_put<8>(G, kColComb + 96 + 8 * c, e);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float m[32];
        read_cols<32>(G, 32 * c, m);
        bias_relu<EB, 32>(m, kL81 + c, rs_main[c], aux);
        tmem_put<32>(G, kColComb + 32 * c, m);
    }
    tc::tmem_wait_st();
    // tail, once per distinct albedo channel (core/radiancePredict.cu:375-419)
    float srv[3] = {sr.x, sr.y, sr.z}, P[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        if (ch == 1 && srv[1] == srv[0]) { P[1] = P[0]; continue; }
        if (ch == 2 && srv[2] == srv[0]) { P[2] = P[0]; continue; }
        if (ch == 2 && srv[2] == srv[1]) { P[2] = P[1]; continue; }
        if (ch > 0) {   // the previous tail's accumulators covered kColHf
            tmem_put<16>(G, kColHf, hf);
            tc::tmem_wait_st();
        }
        TailOut t = tc_tail<EB>(G, st, aux, g, gamma, powf(srv[ch], 4.0f));
        st = t.st;
        P[ch] = t.p;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = fmaxf(expf(P[c]) - 1.0f, 0.0f) * powf(srv[c], 4.0f);
    return st;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
struct TcArgs {
    const uint8_t* wimg;        // operand image (global)
    int wimg_bytes;
    const float* aux;           // fp32 constants of the CUDA-core parts (kAux* layout)
    int* err;
    int* tile_counter;
    // inputs: either row-major features [n][576] + gamma, or staged records
    const float* feat;
    const float* gamma;
    int n;
    float g;
    f3 sr;
    float* out3;                // row-major [n][3]
    // staged records: segs[0, nseg), or seg0 alone when segs is null
    const TcSegment* segs;
    int nseg;
    TcSegment seg0;
};

template <int EB, bool STAGED>
__global__ void __launch_bounds__(kGroups * kGroupThreads, 1) k_mlp_tc(const __grid_constant__ TcArgs A) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int wbytes = (A.wimg_bytes + 1023) & ~1023;
    uint8_t* wimg = smem;
    uint8_t* abuf = smem + wbytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(abuf + kGroups * kABytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + kGroups);
    int* tile_slot = reinterpret_cast<int*>(tslot + 1);
    int* seg_start = tile_slot + kGroups;   // staged: first tile of each segment, [nseg + 1]
    float* aux_s = reinterpret_cast<float*>(seg_start + kTcMaxSegments + 1 + 3);   // 16-byte aligned below
    const TcSegment* segs = A.segs ? A.segs : &A.seg0;
    const int nseg = A.segs ? A.nseg : 1;

    const int tid = threadIdx.x, warp = tid / 32;
    // weights -> shared memory
    for (int i = tid * 16; i < A.wimg_bytes; i += blockDim.x * 16)
        *reinterpret_cast<uint4*>(wimg + i) = __ldg(reinterpret_cast<const uint4*>(A.wimg + i));
    aux_s = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(aux_s) + 15) & ~(uintptr_t)15);
    for (int i = tid * 4; i < kAuxCount; i += blockDim.x * 4)
        *reinterpret_cast<float4*>(aux_s + i) = __ldg(reinterpret_cast<const float4*>(A.aux + i));
    if (warp == 0) {
        tc::tmem_alloc(tslot, kGroups * kTmemColsPerGroup);
        tc::tmem_relinquish();
    }
    if (tid < kGroups) tc::mbar_init(mbar + tid, 1);
    if (STAGED && tid == 32) {
        int acc = 0;
        for (int q = 0; q < nseg; ++q) {
            seg_start[q] = acc;
            acc += (*segs[q].rec_count + 127) / 128;
        }
        seg_start[nseg] = acc;
    }
    tc::mbar_fence_init();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *tslot;

    Group G;
    G.g = tid / kGroupThreads;
    G.t = tid % kGroupThreads;
    G.a_s = tc::smem_addr(abuf + G.g * kABytes);
    G.wimg_s = tc::smem_addr(wimg);
    G.mbar_s = tc::smem_addr(mbar + G.g);
    G.tmem = tbase + (uint32_t)(G.g * kTmemColsPerGroup) + ((uint32_t)(32 * ((tid / 32) % 4)) << 16);
    G.err = A.err;
    int st = 0;

    const int total_tiles = STAGED ? seg_start[nseg] : (A.n + 127) / 128;
    for (;;) {
        if (G.t == 0) tile_slot[G.g] = atomicAdd(A.tile_counter, 1);
        group_bar(G.g);
        int tile = tile_slot[G.g];
        group_bar(G.g);
        if (tile >= total_tiles || (st & kStFailed)) break;
        // staged records from the last tile down: the gather wrote its
        // features in record order just before, so the last tiles' features
        // are still in L2 when the first groups ask for them
        if (STAGED) tile = total_tiles - 1 - tile;
        float o[3];
        if (STAGED) {
            int q = 0;
            while (tile >= seg_start[q + 1]) ++q;
            const TcSegment* S = segs + q;
            const int r = (tile - seg_start[q]) * 128 + G.t;
            const bool valid = r < *S->rec_count;
            const size_t cap = S->rec_cap;
            float gamma = valid ? S->rec_f[15 * cap + r] : 0.0f;
            TileFeatures src{reinterpret_cast<const __half2*>(S->feat) + (size_t)(r >> 5) * 288 * 32 + (r & 31), valid};
            st = tc_network<EB>(G, st, src, aux_s, gamma, S->g, S->sr, o);
            if (valid && !(st & kStFailed)) {
                int pix = S->rec_pix[r];
                f3 hit = mk3(S->rec_f[r], S->rec_f[cap + r], S->rec_f[2 * cap + r]);
                f3 res = mul(mul(mk3(o[0], o[1], o[2]), S->light_color), S->scatter_rate);
                float4 v4 = make_float4(fmaxf(res.x, 0.0f), fmaxf(res.y, 0.0f), fmaxf(res.z, 0.0f),
                                        fmaxf(length(sub(S->ori, hit)), 0.0f));
                const int mean_k = S->mean_k;
                float rate = 1.0f / (float)(1 + mean_k);
                float4 a = mean_k == 0 ? make_float4(0, 0, 0, 0) : S->accum[pix];
                S->accum[pix] = make_float4(lerp(a.x, v4.x, rate), lerp(a.y, v4.y, rate), lerp(a.z, v4.z, rate),
                                            lerp(a.w, v4.w, rate));
            }
        } else {
            const int r = tile * 128 + G.t;
            const bool valid = r < A.n;
            float gamma = valid ? A.gamma[r] : 0.0f;
            RowFeatures src{A.feat + (size_t)r * 576, valid};
            st = tc_network<EB>(G, st, src, aux_s, gamma, A.g, A.sr, o);
            if (valid && !(st & kStFailed)) {
                A.out3[3 * (size_t)r] = o[0];
                A.out3[3 * (size_t)r + 1] = o[1];
                A.out3[3 * (size_t)r + 2] = o[2];
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tbase, kGroups * kTmemColsPerGroup);
    }
}

static size_t tc_smem_bytes(int eb) {
    return (size_t)((image_bytes(eb) + 1023) & ~1023) + kGroups * kABytes + kGroups * 8 + 16 +
           (kTcMaxSegments + 1 + 3) * sizeof(int) + 16 + kAuxCount * sizeof(float);
}

template <int EB, bool STAGED>
static cudaError_t launch_tc(TcArgs& a, int sms, cudaStream_t s) {
    size_t smem = tc_smem_bytes(EB);
    cudaError_t e = cudaFuncSetAttribute(k_mlp_tc<EB, STAGED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.tile_counter, 0, sizeof(int), s)) != cudaSuccess) return e;
    k_mlp_tc<EB, STAGED><<<sms, kGroups * kGroupThreads, smem, s>>>(a);
    return cudaGetLastError();
}

static TcArgs base_args(const TcWeights& w, bool fp8) {
    TcArgs a{};
    a.wimg = (const uint8_t*)(fp8 ? w.d_fp8 : w.d_bf16);
    a.wimg_bytes = image_bytes(fp8 ? 1 : 2);
    a.aux = w.d_aux;
    a.err = w.d_err;
    a.tile_counter = w.d_counter;
    return a;
}

cudaError_t tc_launch_mlp(const TcWeights& w, bool fp8, const float* feat, const float* gamma, float g, const float sr[3],
                          int n, float* out3, int sms, cudaStream_t s) {
    if (!w.ready || !w.d_fp32) return cudaErrorNotReady;
    TcArgs a = base_args(w, fp8);
    a.feat = feat;
    a.gamma = gamma;
    a.n = n;
    a.g = g;
    a.sr = mk3(sr[0], sr[1], sr[2]);
    a.out3 = out3;
    return fp8 ? launch_tc<1, false>(a, sms, s) : launch_tc<2, false>(a, sms, s);
}

cudaError_t tc_launch_mlp_at(const TcWeights& w, bool fp8, const float* feat, const float* gamma, float g,
                             const float sr[3], int n, float* out3, int* tile_counter, int* err, int sms,
                             cudaStream_t s) {
    if (!w.ready || !w.d_fp32 || !tile_counter || !err) return cudaErrorNotReady;
    TcArgs a = base_args(w, fp8);
    a.err = err;
    a.tile_counter = tile_counter;
    a.feat = feat;
    a.gamma = gamma;
    a.n = n;
    a.g = g;
    a.sr = mk3(sr[0], sr[1], sr[2]);
    a.out3 = out3;
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    return fp8 ? launch_tc<1, false>(a, sms, s) : launch_tc<2, false>(a, sms, s);
}

TcSegment tc_segment(const VolumeDev& v, const ViewDev& view, const HitRecords& rec, const float* feat,
                     float4* accum) {
    TcSegment q{};
    q.feat = feat;
    q.rec_count = rec.count;
    q.rec_pix = rec.pix;
    q.rec_f = rec.f;
    q.rec_cap = rec.cap;
    q.accum = accum;
    q.sr = mk3(v.scatter_rate.x / 1.001f, v.scatter_rate.y / 1.001f, v.scatter_rate.z / 1.001f);
    q.light_color = view.light_color;
    q.scatter_rate = v.scatter_rate;
    q.ori = view.ori;
    q.g = view.g;
    q.mean_k = view.mean_k;
    return q;
}

cudaError_t tc_launch_mlp_rec(const TcWeights& w, bool fp8, const VolumeDev& v, const ViewDev& view,
                              const HitRecords& rec, const float* feat, float4* accum, const TcScratch& sc, int sms,
                              cudaStream_t s) {
    if (!w.ready || !w.d_fp32 || !sc.d) return cudaErrorNotReady;
    TcArgs a = base_args(w, fp8);
    a.tile_counter = sc.d;
    a.err = sc.d + 1;
    a.segs = nullptr;
    a.nseg = 1;
    a.seg0 = tc_segment(v, view, rec, feat, accum);
    return fp8 ? launch_tc<1, true>(a, sms, s) : launch_tc<2, true>(a, sms, s);
}

cudaError_t tc_launch_mlp_segments(const TcWeights& w, bool fp8, const TcSegment* d_segs, int nseg,
                                   const TcScratch& sc, int sms, cudaStream_t s) {
    if (!w.ready || !w.d_fp32 || !sc.d || !d_segs) return cudaErrorNotReady;
    if (nseg < 1 || nseg > kTcMaxSegments) return cudaErrorInvalidValue;
    TcArgs a = base_args(w, fp8);
    a.tile_counter = sc.d;
    a.err = sc.d + 1;
    a.segs = d_segs;
    a.nseg = nseg;
    return fp8 ? launch_tc<1, true>(a, sms, s) : launch_tc<2, true>(a, sms, s);
}

// ---------------------------------------------------------------------------
// self-test: one M=128 GEMM D = A * B^T through the same descriptors
// ---------------------------------------------------------------------------
template <int EB>
__global__ void __launch_bounds__(128, 1) k_tc_gemm_test(const float* __restrict__ A, const float* __restrict__ B,
                                                         int n, int k, float* __restrict__ D, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int kp = k;   // multiple of 16 (BF16) / 32 (E4M3)
    uint8_t* sa = smem;
    uint8_t* sb = smem + 128 * kp * EB;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sb + 128 * kp * EB);
    uint32_t* slot = reinterpret_cast<uint32_t*>(mbar + 1);
    int t = threadIdx.x;
    if (t < 32) { tc::tmem_alloc(slot, 128); tc::tmem_relinquish(); }
    if (t == 0) tc::mbar_init(mbar, 1);
    tc::mbar_fence_init();
    for (int idx = t; idx < 128 * kp; idx += 128) {
        int m = idx / kp, kk = idx % kp;
        float va = A[m * k + kk];
        float vb = m < n ? B[m * k + kk] : 0.0f;
        if (EB == 2) {
            uint32_t pa = tc::pack_bf16(va, 0.0f), pb = tc::pack_bf16(vb, 0.0f);
            *reinterpret_cast<unsigned short*>(sa + op_off(m, kk, kp, 2)) = (unsigned short)(pa & 0xFFFF);
            *reinterpret_cast<unsigned short*>(sb + op_off(m, kk, kp, 2)) = (unsigned short)(pb & 0xFFFF);
        } else {
            sa[op_off(m, kk, kp, 1)] = (uint8_t)(tc::pack_e4m3(va, 0.0f) & 0xFF);
            sb[op_off(m, kk, kp, 1)] = (uint8_t)(tc::pack_e4m3(vb, 0.0f) & 0xFF);
        }
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    uint32_t tbase = *slot;
    if (t == 0) {
        uint32_t idesc = tc::instr_desc(128, n, EB == 2 ? tc::kFmtBF16 : tc::kFmtE4M3);
        uint32_t sbo = (uint32_t)(kp * EB * 8);
        for (int s = 0; s < kp * EB / 32; ++s) {
            uint64_t ad = tc::smem_desc(tc::smem_addr(sa) + s * 256, 128, sbo);
            uint64_t bd = tc::smem_desc(tc::smem_addr(sb) + s * 256, 128, sbo);
            if (EB == 2) tc::mma_bf16(tbase, ad, bd, idesc, s > 0);
            else tc::mma_fp8(tbase, ad, bd, idesc, s > 0);
        }
        tc::mma_commit(mbar);
    }
    bool ok = tc::mbar_wait(mbar, 0, kWaitLimit);
    if (!ok && t == 0) atomicExch(err, 1);
    tc::fence_after_sync();
    if (ok) {
        uint32_t lane_addr = tbase + ((uint32_t)(32 * (t / 32)) << 16);
        for (int c0 = 0; c0 < n; c0 += 16) {
            float v[16];
            tc::tmem_ld16(lane_addr + c0, v);
            for (int i = 0; i < 16; ++i) D[t * n + c0 + i] = v[i];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (t < 32) { tc::fence_after_sync(); tc::tmem_dealloc(tbase, 128); }
}

cudaError_t tc_gemm_test(bool fp8, const float* A, const float* B, int n, int k, float* D, int* err, cudaStream_t s) {
    int eb = fp8 ? 1 : 2;
    size_t smem = (size_t)2 * 128 * k * eb + 64;
    cudaError_t e;
    if (fp8) {
        if ((e = cudaFuncSetAttribute(k_tc_gemm_test<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return e;
        k_tc_gemm_test<1><<<1, 128, smem, s>>>(A, B, n, k, D, err);
    } else {
        if ((e = cudaFuncSetAttribute(k_tc_gemm_test<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return e;
        k_tc_gemm_test<2><<<1, 128, smem, s>>>(A, B, n, k, D, err);
    }
    return cudaGetLastError();
}

}  // namespace mrp
