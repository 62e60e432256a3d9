// ref_shim_support.cpp -- definitions behind the CUDA stand-ins of
// shim/ref_prelude.h (thread indices, software texture fetch, curand through
// the build's Philox streams, warp intrinsics), shared by the harnesses of
// the CPU checker build (oracle/_ref).  TEST INFRASTRUCTURE ONLY.
#include "ref_support.h"

thread_local uint3 threadIdx, blockIdx;
thread_local dim3 blockDim, gridDim;

// ---------------------------------------------------------------------------
// software texture helpers used by ref_prelude.h
// ---------------------------------------------------------------------------
float ref_shim_lerp(float a, float b, float v) { return a * (1.0f - v) + b * v; }
float ref_shim_fetch3(const float* d, int nx, int ny, int nz, int x, int y, int z, bool clamp) {
    if (clamp) {
        x = x < 0 ? 0 : (x > nx - 1 ? nx - 1 : x);
        y = y < 0 ? 0 : (y > ny - 1 ? ny - 1 : y);
        z = z < 0 ? 0 : (z > nz - 1 ? nz - 1 : z);
    } else if ((unsigned)x >= (unsigned)nx || (unsigned)y >= (unsigned)ny || (unsigned)z >= (unsigned)nz) {
        return 0.0f;
    }
    return d[((size_t)z * ny + y) * nx + x];
}

// ---------------------------------------------------------------------------
// RNG stand-in: Philox-4x32-10 stream chosen by the harness (same definition
// as the oracle and the kernels: key = (id, seed ^ kind*0x9E3779B9),
// counter = (n/4, sub, frame, kind)).
// ---------------------------------------------------------------------------
thread_local uint32_t t_kind = 0, t_id = 0, t_sub = 0, t_frame = 0, t_seed = 0;
static void philox(const uint32_t c_in[4], const uint32_t k_in[2], uint32_t out[4]) {
    uint32_t c0 = c_in[0], c1 = c_in[1], c2 = c_in[2], c3 = c_in[3], k0 = k_in[0], k1 = k_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1, n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
void curand_init(unsigned long long, unsigned long long, unsigned long long, curandState* s) {
    s->key[0] = t_id;
    s->key[1] = t_seed ^ (t_kind * 0x9E3779B9u);
    s->sub = t_sub; s->frame = t_frame; s->kind = t_kind; s->n = 0;
}
float curand_uniform(curandState* s) {
    uint32_t c[4] = {s->n >> 2, s->sub, s->frame, s->kind}, o[4];
    philox(c, s->key, o);
    uint32_t x = o[s->n & 3];
    s->n++;
    return (float)(((x >> 9) << 1) | 1u) * 5.9604644775390625e-8f;
}
void ref_set_stream(uint32_t kind, uint32_t id, uint32_t sub, uint32_t frame, uint32_t seed) {
    t_kind = kind; t_id = id; t_sub = sub; t_frame = frame; t_seed = seed;
}

// ---------------------------------------------------------------------------
// Warp emulation: the 32 lanes of a warp run as 32 threads; every collective
// publishes into a double-buffered slot and meets at one barrier.  A lane
// rewrites slot k&1 only after barrier k-1, which every lane reaches only
// after reading slot (k-2)&1, so one barrier per collective is enough.
//
// The reference issues __shfl_sync only as weight broadcasts in complete
// source-lane sequences 0, 1, ..., 31 of one unchanged value
// (core/radiancePredict.cu:147-155, 208-222).  A call with src_lane 0 is
// therefore the collective (publish + barrier); calls with src_lane > 0 read
// the slot of that sequence.  The emulation aborts if a lane ever passes a
// value different from the one it published, i.e. if that pattern breaks.
// ---------------------------------------------------------------------------
thread_local Warp* t_warp = nullptr;
thread_local int t_lane = 0, t_phase = 0, t_shfl_slot = -1;
unsigned ref_shim_lane() { return (unsigned)t_lane; }
float __shfl_sync(unsigned, float v, int src, int) {
    if (!t_warp) return v;
    src &= 31;
    if (src == 0) {
        int p = t_phase;
        t_warp->f[p][t_lane] = v;
        t_warp->bar.arrive_and_wait();
        t_shfl_slot = p;
        t_phase ^= 1;
    } else if (t_shfl_slot < 0 || !(t_warp->f[t_shfl_slot][t_lane] == v ||
                                   (v != v && t_warp->f[t_shfl_slot][t_lane] != t_warp->f[t_shfl_slot][t_lane]))) {
        std::fprintf(stderr, "ref_harness: unexpected __shfl_sync pattern\n");
        std::abort();
    }
    return t_warp->f[t_shfl_slot][src];
}
unsigned __ballot_sync(unsigned, int pred) {
    if (!t_warp) return pred ? 1u : 0u;
    int p = t_phase;
    t_warp->u[p][t_lane] = pred ? 1u : 0u;
    t_warp->bar.arrive_and_wait();
    unsigned r = 0;
    for (int l = 0; l < 32; ++l) r |= t_warp->u[p][l] << l;
    t_phase ^= 1;
    return r;
}
void __syncwarp(unsigned) {
    if (t_warp) t_warp->bar.arrive_and_wait();
}
