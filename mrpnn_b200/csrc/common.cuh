// common.cuh -- device building blocks shared by the MRPNN B200 kernels.
//
// Rounding order.  The reference path is float arithmetic whose results the
// build reproduces bit for bit where the operations are +, -, *, /, sqrt and
// comparisons.  nvcc would otherwise contract a*b+c into FMAs, so every
// expression that must keep the reference's rounding is written with the
// IEEE round-to-nearest intrinsics below (which the compiler never fuses).
// Transcendentals (log, exp, pow, atan, acos, sin, cos, tan) use the
// non-fast-math CUDA functions; they can differ from the host's libm in the
// last bit, which the parity tests allow for.
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#define MRP_HD __host__ __device__ __forceinline__
#define MRP_D __device__ __forceinline__

namespace mrp {

// ---------------------------------------------------------------------------
// exact float ops
// ---------------------------------------------------------------------------
MRP_D float fa(float a, float b) { return __fadd_rn(a, b); }
MRP_D float fs(float a, float b) { return __fsub_rn(a, b); }
MRP_D float fm(float a, float b) { return __fmul_rn(a, b); }
MRP_D float fd(float a, float b) { return __fdiv_rn(a, b); }
MRP_D float fsq(float a) { return __fsqrt_rn(a); }

struct f3 { float x, y, z; };
MRP_HD f3 mk3(float x, float y, float z) { return {x, y, z}; }
MRP_D f3 add(f3 a, f3 b) { return {fa(a.x, b.x), fa(a.y, b.y), fa(a.z, b.z)}; }
MRP_D f3 sub(f3 a, f3 b) { return {fs(a.x, b.x), fs(a.y, b.y), fs(a.z, b.z)}; }
MRP_D f3 mul(f3 a, f3 b) { return {fm(a.x, b.x), fm(a.y, b.y), fm(a.z, b.z)}; }
MRP_D f3 mul(f3 a, float b) { return {fm(a.x, b), fm(a.y, b), fm(a.z, b)}; }
MRP_D f3 div(f3 a, float b) { return {fd(a.x, b), fd(a.y, b), fd(a.z, b)}; }
MRP_D f3 adds(f3 a, float b) { return {fa(a.x, b), fa(a.y, b), fa(a.z, b)}; }
MRP_D f3 subs(f3 a, float b) { return {fs(a.x, b), fs(a.y, b), fs(a.z, b)}; }
MRP_D f3 neg(f3 a) { return {-a.x, -a.y, -a.z}; }
// dot(a,b) = a.x*b.x + a.y*b.y + a.z*b.z, left to right (core/vector.cu:22)
MRP_D float dot(f3 a, f3 b) { return fa(fa(fm(a.x, b.x), fm(a.y, b.y)), fm(a.z, b.z)); }
MRP_D f3 normalize(f3 v) { float l = fsq(dot(v, v)); return {fd(v.x, l), fd(v.y, l), fd(v.z, l)}; }
MRP_D f3 cross(f3 a, f3 b) {
    return {fs(fm(a.y, b.z), fm(a.z, b.y)), fs(fm(a.z, b.x), fm(a.x, b.z)), fs(fm(a.x, b.y), fm(a.y, b.x))};
}
MRP_D float length(f3 a) { return fsq(dot(a, a)); }
// lerp(a,b,v) = a*(1-v) + b*v (core/vector.cu:33)
MRP_D float lerp(float a, float b, float v) { return fa(fm(a, fs(1.0f, v)), fm(b, v)); }
MRP_D f3 ld3(const float* p) { return {p[0], p[1], p[2]}; }

// inv / RayBoxOffset / RayBoxDistance (core/vector.cu:19, 46-80)
MRP_D f3 inv(f3 a) {
    return {a.x == 0 ? 999999999.0f : fd(1.0f, a.x), a.y == 0 ? 999999999.0f : fd(1.0f, a.y),
            a.z == 0 ? 999999999.0f : fd(1.0f, a.z)};
}
// ray_box_offset with inv(dir) already taken (for a direction shared by many
// points; same operations after the inverse).
MRP_D float ray_box_offset_inv(f3 p, f3 dir) {
    f3 to_axil = mul(neg(p), dir);
    f3 face = mul(mk3(0.4999f, 0.4999f, 0.4999f), dir);
    f3 d0 = add(to_axil, face), d1 = sub(to_axil, face);
    float tmi = fmaxf(fminf(d0.x, d1.x), fmaxf(fminf(d0.y, d1.y), fminf(d0.z, d1.z)));
    float tma = fminf(fmaxf(d0.x, d1.x), fminf(fmaxf(d0.y, d1.y), fmaxf(d0.z, d1.z)));
    return tma >= tmi ? fmaxf(tmi, 0.0f) : -1.0f;
}
MRP_D float ray_box_offset(f3 p, f3 dir) { return ray_box_offset_inv(p, inv(dir)); }
MRP_D float ray_box_distance(f3 p, f3 dir) {
    dir = inv(dir);
    f3 to_axil = mul(neg(p), dir);
    f3 face = mul(mk3(0.5f, 0.5f, 0.5f), dir);
    f3 d0 = add(to_axil, face), d1 = sub(to_axil, face);
    return fminf(fmaxf(d0.x, d1.x), fminf(fmaxf(d0.y, d1.y), fmaxf(d0.z, d1.z)));
}

// HenyeyGreenstein (core/vector.cu:210-214): (1-g^2)/(1+g^2-2g cos)^1.5 / 4
MRP_D float hg(float c, float g) {
    float g2 = fm(g, g);
    return fm(fd(fs(1.0f, g2), powf(fs(fa(1.0f, g2), fm(fm(2.0f, g), c)), 1.5f)), 0.25f);
}
// SampleHenyeyGreenstein (core/vector.cu:216-242)
MRP_D f3 sample_hg(float e0, float e1, f3 v, float g) {
    float cost;
    if (fabsf(g) < 0.0001) {
        cost = fs(fm(e0, 2.0f), 1.0f);
    } else {
        float g2 = fm(g, g);
        float t0 = fd(fs(1.0f, g2), fa(fs(1.0f, g), fm(fm(2.0f, g), e0)));
        cost = fd(fs(fa(1.0f, g2), fm(t0, t0)), fm(2.0f, g));
    }
    float phi = (float)(2.0 * 3.14159265359 * (double)e1);
    float sint = fsq(fmaxf(0.0f, fs(1.0f, fm(cost, cost))));
    f3 v2 = fabsf(v.z) > 0.70710678118654757 ? normalize(cross(v, mk3(0, 1, 0))) : normalize(cross(v, mk3(0, 0, 1)));
    f3 v3 = cross(v2, v);
    return add(add(mul(v3, fm(sint, cosf(phi))), mul(v2, fm(sint, sinf(phi)))), mul(v, cost));
}
// UniformSampleSphere (core/vector.cu:195-208)
MRP_D f3 uniform_sphere(float ex, float ey) {
    float phi = fm(fm(2.0f, 3.14159265359f), ex);
    float cost = fs(1.0f, fm(2.0f, ey));
    float sint = fsq(fs(1.0f, fm(cost, cost)));
    return {fm(sint, cosf(phi)), fm(sint, sinf(phi)), cost};
}

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  A stream is addressed
// by (kind, id, sub, frame, seed); its n-th uniform is word n%4 of
// Philox(counter = (n/4, sub, frame, kind), key = (id, seed ^ kind*0x9E3779B9)).
// Uniforms are odd multiples of 2^-24, so never 0 and never 1.
// ---------------------------------------------------------------------------
MRP_HD void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
MRP_HD float u01(uint32_t x) { return (float)(((x >> 9) << 1) | 1u) * 5.9604644775390625e-8f; }

enum StreamKind : uint32_t { kPixelStream = 0, kLutStream = 1, kBakeStream = 2, kNeeStream = 3, kSampleStream = 4,
                             kTrStream = 5, kEnvLightStream = 6 };

struct Stream {
    uint32_t k0, k1, sub, frame, kind, n;
    uint32_t blk[4];
    MRP_D Stream(uint32_t kind_, uint32_t id, uint32_t sub_, uint32_t frame_, uint32_t seed)
        : k0(id), k1(seed ^ (kind_ * 0x9E3779B9u)), sub(sub_), frame(frame_), kind(kind_), n(0) {}
    MRP_D void restart() { n = 0; }
    MRP_D float next() {
        if ((n & 3) == 0) philox(n >> 2, sub, frame, kind, k0, k1, blk);
        float r;
        switch (n & 3) { case 0: r = u01(blk[0]); break; case 1: r = u01(blk[1]); break;
                         case 2: r = u01(blk[2]); break; default: r = u01(blk[3]); }
        ++n;
        return r;
    }
};

// ---------------------------------------------------------------------------
// Software linear-filtered fetches with normalized coordinates, standing in
// for tex3D/tex2D (see the oracle for the exact definition): texel coordinate
// u*N - 0.5, fastest axis interpolated first, weights in fp32.
// ---------------------------------------------------------------------------
// Loads of a grid texel as float: fp32 storage, or fp16 storage widened
// (exact: every fp16 value is a float, so a grid stored in fp16 yields the
// same floats as an fp32 grid holding those values).
MRP_D float ldg_f(const float* p) { return __ldg(p); }
MRP_D float ldg_f(const __half* p) { return __half2float(__ldg(p)); }
MRP_D float fetch_border(const float* __restrict__ g, int n, int x, int y, int z) {
    if ((unsigned)x >= (unsigned)n || (unsigned)y >= (unsigned)n || (unsigned)z >= (unsigned)n) return 0.0f;
    return __ldg(g + ((size_t)x * n + y) * n + z);
}
MRP_D float fetch_clamp(const float* __restrict__ g, int n, int x, int y, int z) {
    x = min(max(x, 0), n - 1); y = min(max(y, 0), n - 1); z = min(max(z, 0), n - 1);
    return __ldg(g + ((size_t)x * n + y) * n + z);
}
// lerp with 1 - v computed once by the caller (same operations, same result).
MRP_D float lerp_w(float a, float b, float v, float omv) { return fa(fm(a, omv), fm(b, v)); }
// Trilinear fetch.  The eight texels come from per-axis clamped coordinates
// (so every load is in bounds); border mode then zeroes the texels whose
// unclamped coordinate lies outside [0, n).  Values and the order of the
// seven lerps are those of fetch_border / fetch_clamp above.
template <bool Clamp, class T = float>
MRP_D float tex3(const T* __restrict__ g, int n, f3 pos) {
    f3 uv = adds(pos, 0.5f);
    float nf = (float)n;
    float px = fs(fm(uv.x, nf), 0.5f), py = fs(fm(uv.y, nf), 0.5f), pz = fs(fm(uv.z, nf), 0.5f);
    float flx = floorf(px), fly = floorf(py), flz = floorf(pz);
    int x = (int)flx, y = (int)fly, z = (int)flz;
    float wx = fs(px, flx), wy = fs(py, fly), wz = fs(pz, flz);
    float ox = fs(1.0f, wx), oy = fs(1.0f, wy), oz = fs(1.0f, wz);
    const int nn = n * n;
    float t000, t001, t010, t011, t100, t101, t110, t111;
    if ((unsigned)x < (unsigned)(n - 1) && (unsigned)y < (unsigned)(n - 1) && (unsigned)z < (unsigned)(n - 1)) {
        // footprint inside the grid: the clamps and border selects are no-ops
        const T* b = g + ((size_t)x * n + y) * n + z;
        t000 = ldg_f(b); t001 = ldg_f(b + 1); t010 = ldg_f(b + n); t011 = ldg_f(b + n + 1);
        t100 = ldg_f(b + nn); t101 = ldg_f(b + nn + 1); t110 = ldg_f(b + nn + n); t111 = ldg_f(b + nn + n + 1);
    } else {
        int x0 = min(max(x, 0), n - 1), x1 = min(max(x + 1, 0), n - 1);
        int y0 = min(max(y, 0), n - 1) * n, y1 = min(max(y + 1, 0), n - 1) * n;
        int z0 = min(max(z, 0), n - 1), z1 = min(max(z + 1, 0), n - 1);
        const T* p0 = g + (size_t)x0 * nn;
        const T* p1 = g + (size_t)x1 * nn;
        t000 = ldg_f(p0 + y0 + z0); t001 = ldg_f(p0 + y0 + z1); t010 = ldg_f(p0 + y1 + z0); t011 = ldg_f(p0 + y1 + z1);
        t100 = ldg_f(p1 + y0 + z0); t101 = ldg_f(p1 + y0 + z1); t110 = ldg_f(p1 + y1 + z0); t111 = ldg_f(p1 + y1 + z1);
        if (!Clamp) {
            bool vx0 = (unsigned)x < (unsigned)n, vx1 = (unsigned)(x + 1) < (unsigned)n;
            bool vy0 = (unsigned)y < (unsigned)n, vy1 = (unsigned)(y + 1) < (unsigned)n;
            bool vz0 = (unsigned)z < (unsigned)n, vz1 = (unsigned)(z + 1) < (unsigned)n;
            t000 = vx0 && vy0 && vz0 ? t000 : 0.0f; t001 = vx0 && vy0 && vz1 ? t001 : 0.0f;
            t010 = vx0 && vy1 && vz0 ? t010 : 0.0f; t011 = vx0 && vy1 && vz1 ? t011 : 0.0f;
            t100 = vx1 && vy0 && vz0 ? t100 : 0.0f; t101 = vx1 && vy0 && vz1 ? t101 : 0.0f;
            t110 = vx1 && vy1 && vz0 ? t110 : 0.0f; t111 = vx1 && vy1 && vz1 ? t111 : 0.0f;
        }
    }
    float c00 = lerp_w(t000, t001, wz, oz);
    float c01 = lerp_w(t010, t011, wz, oz);
    float c10 = lerp_w(t100, t101, wz, oz);
    float c11 = lerp_w(t110, t111, wz, oz);
    return lerp_w(lerp_w(c00, c01, wy, oy), lerp_w(c10, c11, wy, oy), wx, ox);
}
// Contracted forms for the stencil gather, whose outputs are features (held
// to 1e-5 relative, not bit for bit): fused multiply-adds in the coordinate
// and lerp arithmetic.  The march keeps the exact forms above -- its
// accept / stop decisions must match the reference's float order.
MRP_D float lerp_fast(float a, float b, float v) { return fmaf(v, b - a, a); }
// n^3 must stay below 2^31 (the pyramid and TR levels: n <= 256): 32-bit
// offsets.  Footprints inside the grid (the common case) skip the clamps and
// the border selects.
// tex3_fast on a padded level (pad_offset): the texel coordinate is clamped
// to [-1, n] per axis, after which every footprint lies inside the padded
// grid, so there is no branch and no per-texel clamp or border select.  The
// value is tex3_fast's: beyond -1 (or n) both texels of an axis hold the same
// margin value, and lerp_fast(a, a, w) = a for every weight, so moving the
// coordinate to the margin (weight 0) changes nothing.
MRP_D float tex3_padded(const float* __restrict__ g, int n, f3 pos) {
    const float nf = (float)n;
    float px = fmaf(pos.x + 0.5f, nf, -0.5f), py = fmaf(pos.y + 0.5f, nf, -0.5f), pz = fmaf(pos.z + 0.5f, nf, -0.5f);
    px = fminf(fmaxf(px, -1.0f), nf);
    py = fminf(fmaxf(py, -1.0f), nf);
    pz = fminf(fmaxf(pz, -1.0f), nf);
    const float flx = floorf(px), fly = floorf(py), flz = floorf(pz);
    const int P = n + 3;
    const int x = (int)flx + 1, y = (int)fly + 1, z = (int)flz + 1;
    const float wx = px - flx, wy = py - fly, wz = pz - flz;
    const float* b = g + (x * P + y) * P + z;
    const int PP = P * P;
    const float t000 = __ldg(b), t001 = __ldg(b + 1), t010 = __ldg(b + P), t011 = __ldg(b + P + 1);
    const float t100 = __ldg(b + PP), t101 = __ldg(b + PP + 1), t110 = __ldg(b + PP + P), t111 = __ldg(b + PP + P + 1);
    const float c00 = lerp_fast(t000, t001, wz), c01 = lerp_fast(t010, t011, wz);
    const float c10 = lerp_fast(t100, t101, wz), c11 = lerp_fast(t110, t111, wz);
    return lerp_fast(lerp_fast(c00, c01, wy), lerp_fast(c10, c11, wy), wx);
}

// Two trilinear fetches at one position from texel pairs (mip_tr): the
// values tex3_fast gives for each array, when the footprint is inside the
// grid (where border and clamp addressing read the same texels); false (and
// nothing read) otherwise.
MRP_D bool tex3_pair_interior(const float2* __restrict__ g, int n, f3 pos, float* a, float* b) {
    float nf = (float)n;
    float px = fmaf(pos.x + 0.5f, nf, -0.5f), py = fmaf(pos.y + 0.5f, nf, -0.5f), pz = fmaf(pos.z + 0.5f, nf, -0.5f);
    float flx = floorf(px), fly = floorf(py), flz = floorf(pz);
    int x = (int)flx, y = (int)fly, z = (int)flz;
    if (!((unsigned)x < (unsigned)(n - 1) && (unsigned)y < (unsigned)(n - 1) && (unsigned)z < (unsigned)(n - 1)))
        return false;
    float wx = px - flx, wy = py - fly, wz = pz - flz;
    const int nn = n * n;
    const float2* q = g + (x * n + y) * n + z;
    const float2 t000 = __ldg(q), t001 = __ldg(q + 1), t010 = __ldg(q + n), t011 = __ldg(q + n + 1);
    const float2 t100 = __ldg(q + nn), t101 = __ldg(q + nn + 1), t110 = __ldg(q + nn + n), t111 = __ldg(q + nn + n + 1);
    {
        float c00 = lerp_fast(t000.x, t001.x, wz), c01 = lerp_fast(t010.x, t011.x, wz);
        float c10 = lerp_fast(t100.x, t101.x, wz), c11 = lerp_fast(t110.x, t111.x, wz);
        *a = lerp_fast(lerp_fast(c00, c01, wy), lerp_fast(c10, c11, wy), wx);
    }
    {
        float c00 = lerp_fast(t000.y, t001.y, wz), c01 = lerp_fast(t010.y, t011.y, wz);
        float c10 = lerp_fast(t100.y, t101.y, wz), c11 = lerp_fast(t110.y, t111.y, wz);
        *b = lerp_fast(lerp_fast(c00, c01, wy), lerp_fast(c10, c11, wy), wx);
    }
    return true;
}

// tex3_padded of both channels of a padded pair array (pad_pair).
MRP_D void tex3_padded_pair(const float2* __restrict__ g, int n, f3 pos, float* a, float* b) {
    const float nf = (float)n;
    float px = fmaf(pos.x + 0.5f, nf, -0.5f), py = fmaf(pos.y + 0.5f, nf, -0.5f), pz = fmaf(pos.z + 0.5f, nf, -0.5f);
    px = fminf(fmaxf(px, -1.0f), nf);
    py = fminf(fmaxf(py, -1.0f), nf);
    pz = fminf(fmaxf(pz, -1.0f), nf);
    const float flx = floorf(px), fly = floorf(py), flz = floorf(pz);
    const int P = n + 3;
    const int x = (int)flx + 1, y = (int)fly + 1, z = (int)flz + 1;
    const float wx = px - flx, wy = py - fly, wz = pz - flz;
    const float2* q = g + (x * P + y) * P + z;
    const int PP = P * P;
    const float2 t000 = __ldg(q), t001 = __ldg(q + 1), t010 = __ldg(q + P), t011 = __ldg(q + P + 1);
    const float2 t100 = __ldg(q + PP), t101 = __ldg(q + PP + 1), t110 = __ldg(q + PP + P), t111 = __ldg(q + PP + P + 1);
    {
        float c00 = lerp_fast(t000.x, t001.x, wz), c01 = lerp_fast(t010.x, t011.x, wz);
        float c10 = lerp_fast(t100.x, t101.x, wz), c11 = lerp_fast(t110.x, t111.x, wz);
        *a = lerp_fast(lerp_fast(c00, c01, wy), lerp_fast(c10, c11, wy), wx);
    }
    {
        float c00 = lerp_fast(t000.y, t001.y, wz), c01 = lerp_fast(t010.y, t011.y, wz);
        float c10 = lerp_fast(t100.y, t101.y, wz), c11 = lerp_fast(t110.y, t111.y, wz);
        *b = lerp_fast(lerp_fast(c00, c01, wy), lerp_fast(c10, c11, wy), wx);
    }
}

// tex3_fast's footprints that touch the grid's edge: clamped texels, and
// under border addressing the ones outside the grid zeroed.  Out of line:
// rare, and it keeps the fetch's common path short in the loops that call it.
template <bool Clamp>
__device__ __noinline__ float tex3_edge(const float* __restrict__ g, int n, int x, int y, int z, float wx, float wy,
                                        float wz) {
    const int nn = n * n;
    int x0 = min(max(x, 0), n - 1) * nn, x1 = min(max(x + 1, 0), n - 1) * nn;
    int y0 = min(max(y, 0), n - 1) * n, y1 = min(max(y + 1, 0), n - 1) * n;
    int z0 = min(max(z, 0), n - 1), z1 = min(max(z + 1, 0), n - 1);
    float t000 = __ldg(g + x0 + y0 + z0), t001 = __ldg(g + x0 + y0 + z1);
    float t010 = __ldg(g + x0 + y1 + z0), t011 = __ldg(g + x0 + y1 + z1);
    float t100 = __ldg(g + x1 + y0 + z0), t101 = __ldg(g + x1 + y0 + z1);
    float t110 = __ldg(g + x1 + y1 + z0), t111 = __ldg(g + x1 + y1 + z1);
    if (!Clamp) {
        bool vx0 = (unsigned)x < (unsigned)n, vx1 = (unsigned)(x + 1) < (unsigned)n;
        bool vy0 = (unsigned)y < (unsigned)n, vy1 = (unsigned)(y + 1) < (unsigned)n;
        bool vz0 = (unsigned)z < (unsigned)n, vz1 = (unsigned)(z + 1) < (unsigned)n;
        t000 = vx0 && vy0 && vz0 ? t000 : 0.0f; t001 = vx0 && vy0 && vz1 ? t001 : 0.0f;
        t010 = vx0 && vy1 && vz0 ? t010 : 0.0f; t011 = vx0 && vy1 && vz1 ? t011 : 0.0f;
        t100 = vx1 && vy0 && vz0 ? t100 : 0.0f; t101 = vx1 && vy0 && vz1 ? t101 : 0.0f;
        t110 = vx1 && vy1 && vz0 ? t110 : 0.0f; t111 = vx1 && vy1 && vz1 ? t111 : 0.0f;
    }
    float c00 = lerp_fast(t000, t001, wz), c01 = lerp_fast(t010, t011, wz);
    float c10 = lerp_fast(t100, t101, wz), c11 = lerp_fast(t110, t111, wz);
    return lerp_fast(lerp_fast(c00, c01, wy), lerp_fast(c10, c11, wy), wx);
}
template <bool Clamp>
MRP_D float tex3_fast(const float* __restrict__ g, int n, f3 pos) {
    float nf = (float)n;
    float px = fmaf(pos.x + 0.5f, nf, -0.5f), py = fmaf(pos.y + 0.5f, nf, -0.5f), pz = fmaf(pos.z + 0.5f, nf, -0.5f);
    float flx = floorf(px), fly = floorf(py), flz = floorf(pz);
    int x = (int)flx, y = (int)fly, z = (int)flz;
    float wx = px - flx, wy = py - fly, wz = pz - flz;
    if (!((unsigned)x < (unsigned)(n - 1) && (unsigned)y < (unsigned)(n - 1) && (unsigned)z < (unsigned)(n - 1)))
        return tex3_edge<Clamp>(g, n, x, y, z, wx, wy, wz);
    const int nn = n * n;
    const float* b = g + (x * n + y) * n + z;
    const float t000 = __ldg(b), t001 = __ldg(b + 1), t010 = __ldg(b + n), t011 = __ldg(b + n + 1);
    const float t100 = __ldg(b + nn), t101 = __ldg(b + nn + 1), t110 = __ldg(b + nn + n), t111 = __ldg(b + nn + n + 1);
    float c00 = lerp_fast(t000, t001, wz), c01 = lerp_fast(t010, t011, wz);
    float c10 = lerp_fast(t100, t101, wz), c11 = lerp_fast(t110, t111, wz);
    return lerp_fast(lerp_fast(c00, c01, wy), lerp_fast(c10, c11, wy), wx);
}

constexpr int kLut = 512;
constexpr int kGtexPairs = 8;   // pair textures of stencil layers 1..7 (index 0 unused)
constexpr int kLutAlloc = kLut * kLut + 160;   // the LUT and its lut_dirs table
MRP_D float tex_lut(const float* __restrict__ lut, float u, float v) {
    float px = fs(fm(u, (float)kLut), 0.5f), py = fs(fm(v, (float)kLut), 0.5f);
    int x = (int)floorf(px), y = (int)floorf(py);
    float wx = fs(px, (float)x), wy = fs(py, (float)y);
    int x0 = min(max(x, 0), kLut - 1), x1 = min(max(x + 1, 0), kLut - 1);
    int y0 = min(max(y, 0), kLut - 1), y1 = min(max(y + 1, 0), kLut - 1);
    float r0 = lerp(__ldg(lut + y0 * kLut + x0), __ldg(lut + y1 * kLut + x0), wy);
    float r1 = lerp(__ldg(lut + y0 * kLut + x1), __ldg(lut + y1 * kLut + x1), wy);
    return lerp(r0, r1, wx);
}

// sum_{i<m} (256>>i)^3 = (2^27 - 2^(27-3m)) / 7 and sum_{i<m} (128>>i)^3 =
// (2^24 - 2^(24-3m)) / 7, both exact in 32 bits for the levels that exist.
MRP_HD size_t mip_offset(int m) { return (size_t)(((1u << 27) - (1u << (27 - 3 * m))) / 7u); }
MRP_HD size_t tr_offset(int m) { return (size_t)(((1u << 24) - (1u << (24 - 3 * m))) / 7u); }
constexpr size_t kMipFloats = 19173961;   // sum_{m<9} (256>>m)^3
constexpr size_t kTrFloats = 2396745;     // sum_{i<8} (128>>i)^3

MRP_D float tex_lut_fast(const float* __restrict__ lut, float u, float v) {
    float px = fmaf(u, (float)kLut, -0.5f), py = fmaf(v, (float)kLut, -0.5f);
    float flx = floorf(px), fly = floorf(py);
    int x = (int)flx, y = (int)fly;
    float wx = px - flx, wy = py - fly;
    float a, b, c, d;   // (x, y), (x, y + 1), (x + 1, y), (x + 1, y + 1)
    if ((unsigned)x < (unsigned)(kLut - 1) && (unsigned)y < (unsigned)(kLut - 1)) {
        const float* p = lut + y * kLut + x;
        a = __ldg(p); b = __ldg(p + kLut); c = __ldg(p + 1); d = __ldg(p + kLut + 1);
    } else {
        int x0 = min(max(x, 0), kLut - 1), x1 = min(max(x + 1, 0), kLut - 1);
        int y0 = min(max(y, 0), kLut - 1) * kLut, y1 = min(max(y + 1, 0), kLut - 1) * kLut;
        a = __ldg(lut + y0 + x0); b = __ldg(lut + y1 + x0); c = __ldg(lut + y0 + x1); d = __ldg(lut + y1 + x1);
    }
    return lerp_fast(lerp_fast(a, b, wy), lerp_fast(c, d, wy), wx);
}

// ---------------------------------------------------------------------------
// Device view of one volume's resources (passed by value to kernels).
// ---------------------------------------------------------------------------
struct VolumeDev {
    const float* density;   // res^3, z fastest (fp32 storage), or null
    const __half* density_h;   // the same grid in fp16 storage, or null
    int res;
    float max_density;
    const float* mips;      // 9 levels (256>>m)^3, concatenated (offsets: mip_offset)
    const float* trs;       // 8 levels (128>>i)^3, concatenated (offsets: tr_offset)
    const float* lut;       // 512x512 HG LUT
    const float* baked;     // NEE transmittance grid
    int baked_res;
    const uint8_t* occ;     // 1 where a brick (or its trilinear apron) holds density != 0
    int occ_shift;          // brick edge = 1 << occ_shift voxels
    const uint8_t* occ2;    // coarse bricks of 4^3 bricks (launch_occupancy_coarse), or null
    int occ2_res;           // coarse bricks per axis
    int occ_res;            // bricks per axis
    f3 scatter_rate;
    float tr_scale;
    f3 sky;
    int nee_mode;           // tracer NEE: 0 baked grid (reference), 1 one Tr() estimate per vertex
    const uint8_t* mip_occ; // occupancy of mip levels 0..kOccMips-1 (8^3 bricks, offsets mip_occ_offset)
    // Box (world coordinates) outside which Density() is exactly 0: the
    // nonzero voxels' bounds grown by the fetch footprint and one voxel more
    // (lo > hi for an all-zero grid); has_bounds = 0 when not computed.
    f3 nz_lo, nz_hi;
    int has_bounds;
    // Padded copies of the small levels (edge 8, 4, 2: mips 5..7, TR levels
    // 4..6) for the stencil gather, or null: see pad_offset / tex3_padded.
    const float* mips_pad;
    const float* trs_pad;
    // Mip level L and TR level L - 1 (same edge, 256 >> L) side by side per
    // texel for L = 1..4 (mip_tr_offset), or null: the gather reads both
    // values of a stencil point with one 8-byte load per texel.
    const float2* mip_tr;
    // The same pairing for the padded levels (mips 5..7 with TR levels 4..6,
    // pad_offset layout, each channel with its own margin), or null.
    const float2* pad_pair;
    // 160 HG-LUT values of the rotated stencil points' own direction (the
    // first LUT factor of X_Hg, which depends only on the point and g), or
    // null; stored right after the LUT (kLutAlloc floats per LUT buffer).
    const float* lut_dirs;
    // Equirect environment map of SetHDRI (RGBA rows of hdri_w texels), or
    // null for the constant sky; env_exp scales it (enviroment_exp).
    const float4* hdri;
    int hdri_w, hdri_h;
    float env_exp;
    // The density grid as a 3D texture (trilinear, border addressing,
    // normalized coordinates) for the frame tracer's free flight, or 0 for
    // the software fetch (mrp_params.tracer_filter).
    cudaTextureObject_t dens_tex;
    // The baked NEE grid as an fp16 texture (trilinear, clamp, normalized
    // coordinates) for the frame tracer's NEE lookup under tracer_filter, as
    // the reference binds it to TR_Mip(0) (core/volume.cu:1687-1693), or 0.
    cudaTextureObject_t baked_tex;
    // The fp16-feature gather through the texture unit's filters
    // (mrp_params.gather_filter), as the reference samples Mip(i), TR_Mip(i)
    // and _HGLut: mip level 0 (trilinear, border) and TR level 0 (trilinear,
    // clamp) for the stencil's layer 0, the (mip L, TR L - 1) pairs of layers
    // 1..7 in one half2 texture each (gtex_alloc_pair: padded, clamp,
    // unnormalized), the HG LUT (bilinear, clamp).  glut_tex 0: the gather
    // filters in software.
    cudaTextureObject_t gmip0_tex, gtr0_tex, gpair_tex[kGtexPairs], glut_tex;
};

// SkyBox (core/render.cuh:24-27): the environment map at u = atan2(-z, x) /
// 2pi + 1/2, v = acos(y) / pi, bilinear with wrap addressing (u interpolated
// first, the order of the reference's host sampler Image_host::Sample,
// core/volume.hpp:35-42), times enviroment_exp; the constant sky when no
// map is set.  Software filtering with fp32 weights (the reference's texture
// unit quantises the weights to 1/256).  The map lookup is an out-of-line
// call: it runs only where a ray leaves the volume, and inlined its
// transcendentals would weigh on the register allocation of the hot loops.
static __device__ __noinline__ f3 sky_map(const float4* __restrict__ hdri, int W, int H, float env_exp, f3 dir) {
    const float u = fa(fm(atan2f(-dir.z, dir.x), (float)(0.5 / 3.1415926)), 0.5f);
    const float t = fm(acosf(fmaxf(fminf(dir.y, 1.0f), -1.0f)), (float)(1.0 / 3.1415926));
    const float px = fs(fm(u, (float)W), 0.5f), py = fs(fm(t, (float)H), 0.5f);
    const float fx = floorf(px), fy = floorf(py);
    const float wx = fs(px, fx), wy = fs(py, fy);
    int x0 = (int)fx % W, y0 = (int)fy % H;
    x0 += x0 < 0 ? W : 0;
    y0 += y0 < 0 ? H : 0;
    const int x1 = x0 + 1 == W ? 0 : x0 + 1, y1 = y0 + 1 == H ? 0 : y0 + 1;
    const float4 a = __ldg(hdri + (size_t)y0 * W + x0), b = __ldg(hdri + (size_t)y0 * W + x1);
    const float4 c = __ldg(hdri + (size_t)y1 * W + x0), d = __ldg(hdri + (size_t)y1 * W + x1);
    const f3 r = mk3(lerp(lerp(a.x, b.x, wx), lerp(c.x, d.x, wx), wy), lerp(lerp(a.y, b.y, wx), lerp(c.y, d.y, wx), wy),
                     lerp(lerp(a.z, b.z, wx), lerp(c.z, d.z, wx), wy));
    return mk3(fm(r.x, env_exp), fm(r.y, env_exp), fm(r.z, env_exp));
}
MRP_D f3 sky_radiance(const VolumeDev& v, f3 dir) {
    return v.hdri ? sky_map(v.hdri, v.hdri_w, v.hdri_h, v.env_exp, dir) : v.sky;
}
// A level of edge n (n <= 8) stored with one texel of margin below and two
// above per axis, (n + 3)^3 floats, texel (x, y, z) at ((x + 1) P + y + 1) P
// + z + 1 (P = n + 3).  The margin holds what the fetch reads outside the
// grid: 0 (border addressing, the density mips) or the nearest edge texel
// (clamp addressing, the TR levels).  Levels of edge 8, 4, 2 in that order.
constexpr int kPadLevelFloats = 11 * 11 * 11 + 7 * 7 * 7 + 5 * 5 * 5;
// Texel offset of level L (1..4) of VolumeDev::mip_tr; L = 5 gives the size.
MRP_HD int mip_tr_offset(int L) { int o = 0; for (int l = 1; l < L; ++l) { int n = 256 >> l; o += n * n * n; } return o; }
MRP_HD int pad_offset(int n) { return n == 8 ? 0 : n == 4 ? 11 * 11 * 11 : 11 * 11 * 11 + 7 * 7 * 7; }

// ---------------------------------------------------------------------------
// Empty-space skipping that keeps every result bit-identical: an 8^3 brick
// is flagged empty only when it and its one-texel apron hold no nonzero
// texel, so any trilinear footprint whose low corner lies in it reads eight
// zeros and the filter returns exactly +0 -- the fetch is skipped, never
// approximated.
// ---------------------------------------------------------------------------
constexpr int kOccMips = 5;   // mip levels 0..4 (256^3 .. 16^3) carry bricks
MRP_HD int mip_occ_offset(int m) { int o = 0; for (int i = 0; i < m; ++i) { int nb = 32 >> i; o += nb * nb * nb; } return o; }
constexpr int kMipOccBytes = 32 * 32 * 32 + 16 * 16 * 16 + 8 * 8 * 8 + 4 * 4 * 4 + 2 * 2 * 2;

// tex3<false> of an n^3 grid with brick flags occ (nb = ceil(n / 8) per
// axis, shift 3); returns 0 without touching the grid for empty bricks.
template <class T>
MRP_D float tex3_occ(const T* __restrict__ g, int n, const uint8_t* __restrict__ occ, int nb, f3 pos) {
    f3 uv = adds(pos, 0.5f);
    float nf = (float)n;
    int x = (int)floorf(fs(fm(uv.x, nf), 0.5f)), y = (int)floorf(fs(fm(uv.y, nf), 0.5f)),
        z = (int)floorf(fs(fm(uv.z, nf), 0.5f));
    if (x < -1 || y < -1 || z < -1 || x > n - 1 || y > n - 1 || z > n - 1) return 0.0f;   // footprint outside
    int b = ((max(x, 0) >> 3) * nb + (max(y, 0) >> 3)) * nb + (max(z, 0) >> 3);
    if (__ldg(occ + b) == 0) return 0.0f;
    return tex3<false>(g, n, pos);
}
// Density() of the full-resolution grid (fp32 or fp16 storage).
MRP_D float density_tex(const VolumeDev& v, f3 p) {
    return v.density_h ? tex3<false>(v.density_h, v.res, p) : tex3<false>(v.density, v.res, p);
}
// The same with the storage type fixed at compile time (DT float: fp32,
// __half: fp16), for the kernels that instantiate one copy per type and so
// keep the test off their inner loops; DT void chooses per call.
template <class DT>
MRP_D float density_as(const VolumeDev& v, f3 p) {
    if constexpr (std::is_same<DT, float>::value) return tex3<false>(v.density, v.res, p);
    else if constexpr (std::is_same<DT, __half>::value) return tex3<false>(v.density_h, v.res, p);
    else return density_tex(v, p);
}
// Density() of the full-resolution grid with its bricks (DT as density_as).
template <class DT = void>
MRP_D float density_occ(const VolumeDev& v, f3 p) {
    if constexpr (std::is_same<DT, float>::value)
        return v.occ ? tex3_occ(v.density, v.res, v.occ, v.occ_res, p) : tex3<false>(v.density, v.res, p);
    else if constexpr (std::is_same<DT, __half>::value)
        return v.occ ? tex3_occ(v.density_h, v.res, v.occ, v.occ_res, p) : tex3<false>(v.density_h, v.res, p);
    else return v.density_h ? density_occ<__half>(v, p) : density_occ<float>(v, p);
}
// Mip level m of the pyramid (256 >> m) at p, with bricks for m < kOccMips.
MRP_D float mip_density(const VolumeDev& v, int m, f3 p) {
    const float* g = v.mips + mip_offset(m);
    int n = 256 >> m;
    if (v.mip_occ && m < kOccMips) return tex3_occ(g, n, v.mip_occ + mip_occ_offset(m), 32 >> m, p);
    return tex3<false>(g, n, p);
}

// ---------------------------------------------------------------------------
// Tr (core/render.cuh:60-103): ratio tracking while tr > 0.5, then delta
// tracking with termination until tr <= 0.001, through the full-resolution
// density.  Both loops share the reference's 10000-iteration bound.
// ---------------------------------------------------------------------------
template <class DT = void>
MRP_D float transmittance(const VolumeDev& v, Stream& st, f3 pos, f3 dir, float dis, float alpha) {
    float smax = fm(v.max_density, alpha);
    float tr = 1.0f, t = 0.0f;
    int loop = 0;
    while (loop++ < 10000 && tr > 0.5) {
        float rk = st.next();
        t = fs(t, fm(fd(logf(fs(1.0f, rk)), smax), v.tr_scale));
        if (t > dis) break;
        float d = density_occ<DT>(v, add(pos, mul(dir, t)));
        float S = fm(d, alpha);
        tr = fm(tr, fs(1.0f, fmaxf(0.0f, fd(S, smax))));
        if (d < 0) t = fs(t, d);
    }
    while (loop++ < 10000 && tr > 0.001) {
        float rk = st.next();
        t = fs(t, fm(fd(logf(fs(1.0f, rk)), smax), v.tr_scale));
        if (t > dis) break;
        float d = density_occ<DT>(v, add(pos, mul(dir, t)));
        float S = fm(d, alpha);
        if (st.next() < fmaxf(0.0f, fd(S, smax))) { tr = 0.0f; break; }
        if (d < 0) t = fs(t, d);
    }
    return tr;
}


// One camera launch (RenderCamera's arguments, core/volume.cu:199).
struct ViewDev {
    int width, height;
    f3 ori, up, right, light_dir, light_color;
    float alpha, g;
    int multi_scatter, spp;
    uint32_t seed;
    int frame;         // RNG launch index ("randNum")
    int mean_k;        // running-mean index of this launch ("frameNum")
    float pass_rate;   // exp(-(2/res) * max_density * alpha), host libm (DeterminateEstimatedHit)
    unsigned long long* counters;   // optional work counters (see launch_hit / launch_trace), else null
    // explicit rays instead of the camera (GetRadiances): ray q = pixel q of a
    // width x 1 launch, origin ray_ori[3q..], direction ray_dir[3q..]
    const float* ray_ori;
    const float* ray_dir;
    // interactive frames (VolumeRender::Render(float3*, Histogram*, ...)):
    // cam_mode 1 uses that kernel's v = (row + r) / H instead of
    // RenderCamera<float4>'s 1 - (row + r) / H; checker renders only the
    // pixels with (row + col + flip) even
    int cam_mode, checker, flip;
};

// Camera ray of pixel (row, col): jitter = the first two draws of the pixel
// stream (RenderCamera, core/volume.cu:208-216 and 67-81).
MRP_D f3 camera_ray_dir(const ViewDev& w, int row, int col) {
    Stream st(kPixelStream, (uint32_t)(row * w.width + col), 0, (uint32_t)w.frame, w.seed);
    float r0 = st.next(), r1 = st.next();
    float u = fs(1.0f, fd(fa((float)col, r0), (float)w.width));
    float vq = fd(fa((float)row, r1), (float)w.height);
    float vv = w.cam_mode ? vq : fs(1.0f, vq);
    f3 fwd = normalize(neg(w.ori));
    f3 d = add(add(fwd, mul(w.right, fs(fm(u, 2.0f), 1.0f))), mul(w.up, fs(fm(vv, 2.0f), 1.0f)));
    return normalize(d);
}
MRP_D bool pixel_selected(const ViewDev& w, int row, int col) { return !w.checker || ((row + col + w.flip) & 1) == 0; }

// Per-thread work tally, flushed to ViewDev::counters once per thread.
struct Tally {
    uint32_t steps = 0, fetches = 0, lookups = 0, events = 0;
};
MRP_D void flush_tally(unsigned long long* c, const Tally& t) {
    atomicAdd(c + 0, (unsigned long long)t.steps);
    atomicAdd(c + 1, (unsigned long long)t.fetches);
    atomicAdd(c + 2, (unsigned long long)t.lookups);
    atomicAdd(c + 3, (unsigned long long)t.events);
}

// ---------------------------------------------------------------------------
// Packed MLP weight layout (fp32, one buffer).  Per SE block: the gate MLP
// 8->8 (no bias) and 8->3 (no bias), then the three branch layers w->w with
// biases in channel order density, TR, HG.  Then the three final 32->32
// (main) or 8->8 (direct-illumination) layers, then the tail.  Names follow
// core/NNWeight.cuh.
// ---------------------------------------------------------------------------
constexpr int kMainW[8] = {8, 8, 16, 16, 16, 32, 32, 32};
constexpr int kMainFrom[8] = {0, 8, 16, 32, 48, 64, 96, 128};
constexpr bool kMainWiden[8] = {false, true, false, false, true, false, false, false};
constexpr int kDiFrom[4] = {160, 168, 176, 184};
constexpr int block_size(int w) { return 64 + 24 + 3 * (w * w + w); }
constexpr int main_block_off(int k) { int o = 0; for (int i = 0; i < k; ++i) o += block_size(kMainW[i]); return o; }
constexpr int kMainFinalOff = main_block_off(8);
constexpr int kDiOff = kMainFinalOff + 3 * (32 * 32 + 32);
constexpr int di_block_off(int k) { return kDiOff + k * block_size(8); }
constexpr int kDiFinalOff = di_block_off(4);
constexpr int kTailOff = kDiFinalOff + 3 * (64 + 8);
constexpr int kLGGSW = kTailOff, kLGGSB = kLGGSW + 24, kLSEFin1W = kLGGSB + 8, kLSEFin2W = kLSEFin1W + 1200;
constexpr int kLC0W = kLSEFin2W + 96, kLC0B = kLC0W + 16384, kLC1W = kLC0B + 128, kLC1B = kLC1W + 8192;
constexpr int kLC2W = kLC1B + 64, kLC2B = kLC2W + 2048, kLXW = kLC2B + 32, kLXB = kLXW + 512;
constexpr int kLXk = kLXB + 16;   // LX0W, LX0B, ..., LX11W, LX11B (256 + 16 each)
constexpr int lxw(int k) { return kLXk + k * 272; }
constexpr int lxb(int k) { return kLXk + k * 272 + 256; }
constexpr int kLX12W = kLXk + 12 * 272, kLX12B = kLX12W + 16;
constexpr int kWeightCount = kLX12B + 1;
static_assert(kWeightCount == 49673, "packed weight count must match core/NNWeight.cuh");
// The device copy appends two transposed copies for the FP32 network:
// LC1W as [128][64] and LSEFin1W as [75][16] (16-byte aligned rows).
constexpr int kLC1T = (kWeightCount + 3) / 4 * 4;
constexpr int kFin1T = kLC1T + 8192;
constexpr int kWeightCountDev = kFin1T + 1200;
static_assert(kLC1T % 4 == 0 && kFin1T % 4 == 0 && kLC0W % 4 == 0 && kLC2W % 4 == 0 && kLXW % 4 == 0 &&
                  kMainFinalOff % 4 == 0 && kDiOff % 4 == 0 && kLXk % 4 == 0,
              "rows read as float4 start on 16-byte boundaries");

}  // namespace mrp
