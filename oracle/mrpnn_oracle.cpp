// mrpnn_oracle.cpp -- CPU restatement of the MRPNN render path.
//
// TEST INFRASTRUCTURE ONLY (see mrpnn_oracle.h).  The product is the CUDA
// library in mrpnn_b200/; this file is the checker it is compared against.
//
// Every function cites the reference file:line it restates.  Float
// expressions keep the reference's evaluation order (the file is built with
// -ffp-contract=off), so results are reproducible to the bit on one machine.
#include "mrpnn_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// float3 maths, core/vector.cu:3-45 (operator order preserved)
// ---------------------------------------------------------------------------
struct f3 { float x, y, z; };
inline f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline f3 operator*(f3 a, float b) { return {a.x * b, a.y * b, a.z * b}; }
inline f3 operator/(f3 a, float b) { return {a.x / b, a.y / b, a.z / b}; }
inline f3 adds(f3 a, float b) { return {a.x + b, a.y + b, a.z + b}; }
inline f3 subs(f3 a, float b) { return {a.x - b, a.y - b, a.z - b}; }
inline f3 neg(f3 a) { return {-a.x, -a.y, -a.z}; }
inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline f3 normalize(f3 v) { float len = std::sqrt(dot(v, v)); return {v.x / len, v.y / len, v.z / len}; }
inline f3 cross(f3 a, f3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float length(f3 a) { return std::sqrt(dot(a, a)); }
inline float lerpf(float a, float b, float v) { return a * (1.0f - v) + b * v; }   // vector.cu:33
inline f3 load3(const float* p) { return {p[0], p[1], p[2]}; }
inline void store3(float* p, f3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
inline float fmin_(float a, float b) { return std::fmin(a, b); }
inline float fmax_(float a, float b) { return std::fmax(a, b); }

// inv(), core/vector.cu:19
inline f3 inv(f3 a) {
    return {a.x == 0 ? 999999999.0f : 1 / a.x, a.y == 0 ? 999999999.0f : 1 / a.y,
            a.z == 0 ? 999999999.0f : 1 / a.z};
}
// RayBoxOffset, core/vector.cu:46-63
float ray_box_offset(f3 p, f3 dir) {
    dir = inv(dir);
    f3 bmax = {0.4999f, 0.4999f, 0.4999f};
    f3 to_axil = neg(p) * dir;
    f3 axil_face = bmax * dir;
    f3 d0 = to_axil + axil_face, d1 = to_axil - axil_face;
    f3 tmin = {fmin_(d0.x, d1.x), fmin_(d0.y, d1.y), fmin_(d0.z, d1.z)};
    f3 tmax = {fmax_(d0.x, d1.x), fmax_(d0.y, d1.y), fmax_(d0.z, d1.z)};
    float tmi = fmax_(tmin.x, fmax_(tmin.y, tmin.z));
    float tma = fmin_(tmax.x, fmin_(tmax.y, tmax.z));
    return tma >= tmi ? fmax_(tmi, 0.0f) : -1.0f;
}
// RayBoxDistance, core/vector.cu:65-80
float ray_box_distance(f3 p, f3 dir) {
    dir = inv(dir);
    f3 bmax = {0.5f, 0.5f, 0.5f};
    f3 to_axil = neg(p) * dir;
    f3 axil_face = bmax * dir;
    f3 d0 = to_axil + axil_face, d1 = to_axil - axil_face;
    f3 tmax = {fmax_(d0.x, d1.x), fmax_(d0.y, d1.y), fmax_(d0.z, d1.z)};
    return fmin_(tmax.x, fmin_(tmax.y, tmax.z));
}
// HenyeyGreenstein, core/vector.cu:210-214 (0.25 factor, i.e. pi x the phase)
float hg(float c, float g) {
    float g2 = g * g;
    return ((1.0f - g2) / std::pow((1.0f + g2 - 2.0f * g * c), 1.5f)) * 0.25f;
}
// SampleHeneyGreenstein / SampleHenyeyGreenstein, core/vector.cu:216-242
float sample_hg_cos(float s, float g) {
    if (std::fabs(g) < 0.0001) return s * 2.0f - 1.0f;
    float g2 = g * g;
    float t0 = (1 - g2) / (1 - g + 2 * g * s);
    return (1 + g2 - t0 * t0) / (2 * g);
}
f3 sample_hg(float e0, float e1, f3 v, float g) {
    float cost = sample_hg_cos(e0, g);
    float phi = (float)(2 * 3.14159265359 * e1);
    float sint = std::sqrt(fmax_(0.0f, 1.0f - cost * cost));
    f3 v2;
    if (std::fabs(v.z) > std::sqrt(0.5)) v2 = normalize(cross(v, f3{0, 1, 0}));
    else v2 = normalize(cross(v, f3{0, 0, 1}));
    f3 v3 = cross(v2, v);
    return (v3 * (sint * std::cos(phi))) + (v2 * (sint * std::sin(phi))) + (v * cost);
}
// UniformSampleSphere, core/vector.cu:195-208
f3 uniform_sphere(float ex, float ey) {
    float phi = 2 * 3.14159265359f * ex;
    float cost = 1 - 2 * ey;
    float sint = std::sqrt(1 - cost * cost);
    return {sint * std::cos(phi), sint * std::sin(phi), cost};
}

// ---------------------------------------------------------------------------
// RNG.  The reference draws from curand XORWOW (core/render.cuh:49-58); the
// build replaces it with counter-based Philox-4x32-10 (Salmon, Moraes, Dror,
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11) so that every
// draw is addressed by (kind, id, sub, frame, seed, n) rather than by thread.
// ---------------------------------------------------------------------------
void philox(const uint32_t c_in[4], const uint32_t k_in[2], uint32_t out[4]) {
    uint32_t c0 = c_in[0], c1 = c_in[1], c2 = c_in[2], c3 = c_in[3];
    uint32_t k0 = k_in[0], k1 = k_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
inline float u01(uint32_t x) {   // odd multiples of 2^-24: never 0, never 1
    return (float)(((x >> 9) << 1) | 1u) * 5.9604644775390625e-8f;
}
struct Stream {
    uint32_t key[2];
    uint32_t sub, frame, kind, n;
    uint32_t block[4];
    uint32_t have = 0xFFFFFFFFu;
    Stream(uint32_t kind_, uint32_t id, uint32_t sub_, uint32_t frame_, uint32_t seed)
        : sub(sub_), frame(frame_), kind(kind_), n(0) {
        key[0] = id;
        key[1] = seed ^ (kind_ * 0x9E3779B9u);
    }
    void restart() { n = 0; have = 0xFFFFFFFFu; }
    float next() {
        uint32_t blk = n >> 2;
        if (blk != have) {
            uint32_t c[4] = {blk, sub, frame, kind};
            philox(c, key, block);
            have = blk;
        }
        return u01(block[n++ & 3]);
    }
};

// ---------------------------------------------------------------------------
// Software texture fetch, standing in for tex3D/tex2D with normalized
// coordinates and linear filtering (bindings: core/volume.cu:1456-1462,
// 1517-1522, 1413-1418, 1655-1660).  Texel coordinate = u*N - 0.5; the lerp
// order (fastest axis innermost) follows the reference's own CPU sampler
// Sample(), core/volume.cu:845-863.  Weights are exact fp32 (the hardware
// quantises them to 1/256).
// ---------------------------------------------------------------------------
inline float fetch(const float* g, int n, int x, int y, int z, bool clamp) {
    if (clamp) {
        x = std::min(std::max(x, 0), n - 1);
        y = std::min(std::max(y, 0), n - 1);
        z = std::min(std::max(z, 0), n - 1);
    } else if ((unsigned)x >= (unsigned)n || (unsigned)y >= (unsigned)n || (unsigned)z >= (unsigned)n) {
        return 0.0f;
    }
    return g[((size_t)x * n + y) * n + z];
}
// pos is the world position (unit box centred at the origin), x slowest.
float tex3(const float* g, int n, f3 pos, bool clamp) {
    f3 uv = adds(pos, 0.5f);
    float nf = (float)n;
    float px = uv.x * nf - 0.5f, py = uv.y * nf - 0.5f, pz = uv.z * nf - 0.5f;
    int x = (int)std::floor(px), y = (int)std::floor(py), z = (int)std::floor(pz);
    float wx = px - (float)x, wy = py - (float)y, wz = pz - (float)z;
    float c00 = lerpf(fetch(g, n, x, y, z, clamp), fetch(g, n, x, y, z + 1, clamp), wz);
    float c01 = lerpf(fetch(g, n, x, y + 1, z, clamp), fetch(g, n, x, y + 1, z + 1, clamp), wz);
    float c10 = lerpf(fetch(g, n, x + 1, y, z, clamp), fetch(g, n, x + 1, y, z + 1, clamp), wz);
    float c11 = lerpf(fetch(g, n, x + 1, y + 1, z, clamp), fetch(g, n, x + 1, y + 1, z + 1, clamp), wz);
    return lerpf(lerpf(c00, c01, wy), lerpf(c10, c11, wy), wx);
}
// 512x512 HG LUT, clamp addressing; v (row) interpolated first, then u.
constexpr int LUT = 512;
float tex_lut(const float* lut, float u, float v) {
    float px = u * (float)LUT - 0.5f, py = v * (float)LUT - 0.5f;
    int x = (int)std::floor(px), y = (int)std::floor(py);
    float wx = px - (float)x, wy = py - (float)y;
    int x0 = std::min(std::max(x, 0), LUT - 1), x1 = std::min(std::max(x + 1, 0), LUT - 1);
    int y0 = std::min(std::max(y, 0), LUT - 1), y1 = std::min(std::max(y + 1, 0), LUT - 1);
    float r0 = lerpf(lut[y0 * LUT + x0], lut[y1 * LUT + x0], wy);
    float r1 = lerpf(lut[y0 * LUT + x1], lut[y1 * LUT + x1], wy);
    return lerpf(r0, r1, wx);
}

const float* mip_ptr(const float* mips, int m) {
    size_t off = 0;
    for (int i = 0; i < m; ++i) { size_t r = 256 >> i; off += r * r * r; }
    return mips + off;
}
const float* tr_ptr(const float* tr, int m) {
    size_t off = 0;
    for (int i = 0; i < m; ++i) { size_t r = 128 >> i; off += r * r * r; }
    return tr + off;
}

// Density(), core/render.cuh:34-38 (full-resolution grid, border addressing)
inline float density(const orc_scene* s, f3 p) { return tex3(s->density, s->res, p, false); }

// ---------------------------------------------------------------------------
// Model file: "MRPNNMD1", u32 count, then {u16 name_len, name, u32 n, f32[n]}.
// ---------------------------------------------------------------------------
std::map<std::string, std::vector<float>> g_model;
const float* T(const char* name) {
    auto it = g_model.find(name);
    if (it == g_model.end()) { std::fprintf(stderr, "oracle: missing tensor %s\n", name); std::abort(); }
    return it->second.data();
}

// ---------------------------------------------------------------------------
// Stencil, GetSamples23_ (core/vector.cu:304-405) and SphereRandom3
// (core/vector.cu:265-302; the unit directions are read from the model file).
// ---------------------------------------------------------------------------
struct StencilEntry { float offset; float layer; int type; int localindex; };
StencilEntry stencil(int index) {
    const float scale = 0.6f;
    auto e = [](float off, float layer, int type, int li) { return StencilEntry{off, layer, type, li}; };
    if (index < 8) { float o = (float)(1.0 / 256.0); o *= lerpf(scale, 1.0f, 1.0f); return e(o, 0.0f, 5, index); }
    if (index < 16) { float o = (float)(2.5 / 256.0); o *= lerpf(scale, 1.0f, 0.8f); return e(o, 1.0f, 5, 8); }
    if (index < 32) { float o = (float)(5.5 / 256.0); o *= lerpf(scale, 1.0f, 0.6f); return e(o, 2.0f, 5, 8); }
    if (index < 48) { float o = (float)(11.5 / 256.0); o *= lerpf(scale, 1.0f, 0.4f); return e(o, 3.0f, 5, 8); }
    if (index < 64) { float o = (float)(23.5 / 256.0); o *= lerpf(scale, 1.0f, 0.2f); return e(o, 4.0f, 5, 8); }
    if (index < 96) { float o = (float)(47.5 / 256.0); o *= scale; return e(o, 5.0f, 5, 8); }
    if (index < 128) { float o = (float)(95.5 / 256.0); o *= scale; return e(o, 6.0f, 5, 8); }
    if (index < 160) { float o = (float)(191.5 / 256.0); o *= scale; return e(o, 7.0f, 5, 8); }
    if (index < 168) { int i = index - 160; float o = (float)(i + 1); o = (float)(o / 256.0); return e(o, 0.0f, 1, 8); }
    if (index < 176) { int i = index - 168; float o = (float)(8.5 + 1 + 2.0 * i); o = (float)(o / 256.0); return e(o, 1.0f, 1, 8); }
    if (index < 184) { int i = index - 176; float o = (float)(26.5 + 4.0 * i); o = (float)(o / 256.0); return e(o, 2.0f, 1, 8); }
    if (index < 192) { int i = index - 184; float o = (float)(60.5 + 8.0 * i); o = (float)(o / 256.0); return e(o, 3.0f, 1, 8); }
    return e(0.0f, 0.0f, 1, 8);
}

// ---------------------------------------------------------------------------
// MLP, RadiancePredictInternal (core/radiancePredict.cu:301-422).
//
// The reference writes the network as SE / SERES / ADD3 / REP3 macros over
// aliased buffers.  Restated as a list of blocks: each block reads the slice
// [from, from+w) of the three feature channels, forms a per-block SE gate
// from their (avg, max) pools plus (g, gamma), feeds
//     in_c = X_c[slice] * gate_c + prev_c          (c = density, TR, HG)
// through relu(W_c in_c + b_c), and then either adds the raw slice (ADD3)
// or, for the two widening blocks, concatenates it (REP3) so the next block
// sees a residual twice as wide.
// ---------------------------------------------------------------------------
struct Block { int from, w, pid; bool widen; const char *sew0, *sew1, *wd, *wt, *wh; };
const Block kMain[8] = {
    {0, 8, 0, false, "LSE01W", "LSE02W", "L01", "L_Tr01", "L_Hg01"},
    {8, 8, 3, true, "LSE11W", "LSE12W", "L11", "L_Tr11", "L_Hg11"},
    {16, 16, 6, false, "LSE21W", "LSE22W", "L21", "L_Tr21", "L_Hg21"},
    {32, 16, 9, false, "LSE31W", "LSE32W", "L31", "L_Tr31", "L_Hg31"},
    {48, 16, 12, true, "LSE41W", "LSE42W", "L41", "L_Tr41", "L_Hg41"},
    {64, 32, 15, false, "LSE51W", "LSE52W", "L51", "L_Tr51", "L_Hg51"},
    {96, 32, 18, false, "LSE61W", "LSE62W", "L61", "L_Tr61", "L_Hg61"},
    {128, 32, 21, false, "LSE71W", "LSE72W", "L71", "L_Tr71", "L_Hg71"},
};
const Block kDI[4] = {
    {160, 8, 24, false, "LDSE01W", "LDSE02W", "LD01", "LD_Tr01", "LD_Hg01"},
    {168, 8, 27, false, "LDSE11W", "LDSE12W", "LD11", "LD_Tr11", "LD_Hg11"},
    {176, 8, 30, false, "LDSE21W", "LDSE22W", "LD21", "LD_Tr21", "LD_Hg21"},
    {184, 8, 33, false, "LDSE31W", "LDSE32W", "LD31", "LD_Tr31", "LD_Hg31"},
};

template <class R> R sigmoid(R o);
template <> float sigmoid<float>(float o) { return (float)(1.0 / (1.0 + (double)std::exp(-o))); }  // :84
template <> double sigmoid<double>(double o) { return 1.0 / (1.0 + std::exp(-o)); }

// out[i] = b[i] + sum_j in[j] W[i*from + j]  (LinearReLU<Size>, LinearReLU_SFL: bias first)
template <class R> void lin_bias_first(const R* in, const float* W, const float* b, int from, int to, R* out) {
    for (int i = 0; i < to; ++i) {
        R acc = (R)b[i];
        for (int j = 0; j < from; ++j) acc += in[j] * (R)W[j + i * from];
        out[i] = acc >= 0 ? acc : (R)0;
    }
}
// LinearReLU(In, Out, From, To, ...) non-template: sum first, bias last (:41-56)
template <class R> void lin_bias_last(const R* in, const float* W, const float* b, int from, int to, R* out) {
    for (int i = 0; i < to; ++i) {
        R acc = 0;
        for (int j = 0; j < from; ++j) acc += in[j] * (R)W[j + i * from];
        acc += (R)b[i];
        out[i] = acc >= 0 ? acc : (R)0;
    }
}
// LinearReLU_Unbias / LinearSm_Unbias (:58-86)
template <class R> void lin_nobias(const R* in, const float* W, int from, int to, R* out, bool sig) {
    for (int i = 0; i < to; ++i) {
        R acc = 0;
        for (int j = 0; j < from; ++j) acc += in[j] * (R)W[j + i * from];
        out[i] = sig ? sigmoid<R>(acc) : (acc >= 0 ? acc : (R)0);
    }
}
std::string wname(const char* base, char kind) { return std::string(base) + kind; }

template <class R>
void mlp_one(const float* feat, float gamma_f, float g_f, const float sr[3], R out[3]) {
    const R g = (R)g_f, gamma = (R)gamma_f;
    R X[3][192];
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < 192; ++i) X[c][i] = (R)feat[c * 192 + i];
    R pool[75];
    pool[72] = g;
    pool[73] = gamma;

    // SE gate, SE/SERES macros lines 1-7 (core/radiancePredict.cu:240-247)
    auto gate = [&](const Block& b, R gates[3]) {
        R p8[8];
        for (int c = 0; c < 3; ++c) {
            R sum = 0, mx = (R)-10000.0;
            for (int i = 0; i < b.w; ++i) { sum += X[c][b.from + i]; mx = std::max(mx, X[c][b.from + i]); }
            sum /= (R)b.w;
            pool[b.pid + c] = sum;
            pool[36 + b.pid + c] = mx;
            p8[c] = sum;
            p8[3 + c] = mx;
        }
        p8[6] = g;
        p8[7] = gamma;
        R h[8];
        lin_nobias<R>(p8, T(b.sew0), 8, 8, h, false);
        lin_nobias<R>(h, T(b.sew1), 8, 3, gates, true);
    };
    // One block over the three channels; prev[c] has width w (or 0 for none).
    auto run_block = [&](const Block& b, R prev[3][32], bool has_prev, R nxt[3][32]) {
        R gates[3];
        gate(b, gates);
        for (int c = 0; c < 3; ++c) {
            R in[32], o[32];
            for (int i = 0; i < b.w; ++i) {
                in[i] = X[c][b.from + i] * gates[c];
                if (has_prev) in[i] = in[i] + prev[c][i];
            }
            const char* base = c == 0 ? b.wd : (c == 1 ? b.wt : b.wh);
            lin_bias_first<R>(in, T(wname(base, 'W').c_str()), T(wname(base, 'B').c_str()), b.w, b.w, o);
            if (b.widen) {   // REP3: next residual = concat(out, raw slice)
                for (int i = 0; i < b.w; ++i) { nxt[c][i] = o[i]; nxt[c][b.w + i] = X[c][b.from + i]; }
            } else {         // ADD3
                for (int i = 0; i < b.w; ++i) nxt[c][i] = o[i] + X[c][b.from + i];
            }
        }
    };

    R comb[128];
    {   // main branch over X[0:160]
        R a[3][32], bb[3][32];
        run_block(kMain[0], a, false, bb);
        for (int k = 1; k < 8; ++k) {
            std::memcpy(a, bb, sizeof(a));
            run_block(kMain[k], a, true, bb);
        }
        const char* last[3] = {"L81", "L_Tr81", "L_Hg81"};
        for (int c = 0; c < 3; ++c)
            lin_bias_first<R>(bb[c], T(wname(last[c], 'W').c_str()), T(wname(last[c], 'B').c_str()), 32, 32, comb + 32 * c);
    }
    {   // direct-illumination branch over X[160:192]
        R a[3][32], bb[3][32];
        run_block(kDI[0], a, false, bb);
        for (int k = 1; k < 4; ++k) {
            std::memcpy(a, bb, sizeof(a));
            run_block(kDI[k], a, true, bb);
        }
        const char* last[3] = {"LD41", "LD_Tr41", "LD_Hg41"};
        for (int c = 0; c < 3; ++c)
            lin_bias_first<R>(bb[c], T(wname(last[c], 'W').c_str()), T(wname(last[c], 'B').c_str()), 8, 8, comb + 96 + 8 * c);
    }

    // Tail SC(p), core/radiancePredict.cu:375-409, once per distinct albedo channel.
    auto tail = [&](float sigma4) -> R {
        pool[74] = (R)sigma4;
        R x[128], y[128], z[16];
        for (int i = 0; i < 120; ++i) x[i] = comb[i];
        lin_bias_last<R>(pool + 72, T("LGGSW"), T("LGGSB"), 3, 8, x + 120);
        R hf[16], gf[6];
        lin_nobias<R>(pool, T("LSEFin1W"), 75, 16, hf, false);
        lin_nobias<R>(hf, T("LSEFin2W"), 16, 6, gf, true);
        const int seg_from[6] = {0, 32, 64, 96, 104, 112}, seg_len[6] = {32, 32, 32, 8, 8, 8};
        for (int s = 0; s < 6; ++s)
            for (int i = 0; i < seg_len[s]; ++i) x[seg_from[s] + i] *= gf[s];
        lin_bias_first<R>(x, T("LC0W"), T("LC0B"), 128, 128, y);
        lin_bias_first<R>(y, T("LC1W"), T("LC1B"), 128, 64, x);
        lin_bias_first<R>(x, T("LC2W"), T("LC2B"), 64, 32, y);
        lin_bias_first<R>(y, T("LXW"), T("LXB"), 32, 16, x);
        char wn[16], bn[16];
        for (int k = 0; k < 6; ++k) {
            std::snprintf(wn, sizeof wn, "LX%dW", 2 * k); std::snprintf(bn, sizeof bn, "LX%dB", 2 * k);
            lin_bias_first<R>(x, T(wn), T(bn), 16, 16, y);
            std::snprintf(wn, sizeof wn, "LX%dW", 2 * k + 1); std::snprintf(bn, sizeof bn, "LX%dB", 2 * k + 1);
            lin_bias_first<R>(y, T(wn), T(bn), 16, 16, z);
            for (int i = 0; i < 16; ++i) x[i] = x[i] + z[i];
        }
        R o;
        lin_bias_last<R>(x, T("LX12W"), T("LX12B"), 16, 1, &o);
        return o;
    };
    // srp = pow(scatterrate, 4) (:324), channel reuse (:411-419)
    R srp[3];
    for (int c = 0; c < 3; ++c) srp[c] = (R)std::pow((R)sr[c], (R)4.0);
    R P[3];
    P[0] = tail((float)srp[0]);
    if (sr[1] == sr[0]) P[1] = P[0]; else P[1] = tail((float)srp[1]);
    if (sr[2] == sr[0]) P[2] = P[0]; else if (sr[2] == sr[1]) P[2] = P[1]; else P[2] = tail((float)srp[2]);
    for (int c = 0; c < 3; ++c) {   // max(exp(P) - 1, 0) * srp  (:421)
        R e = std::exp(P[c]) - (R)1.0;
        out[c] = std::max(e, (R)0) * srp[c];
    }
}

// SkyBox, core/render.cuh:24-27: the equirect environment map at
// u = atan2(-z, x) / 2pi + 1/2, v = acos(y) / pi, filtered bilinearly with
// wrap addressing (u interpolated first, as the reference's own host sampler
// Image_host::Sample, core/volume.hpp:35-42), times enviroment_exp; with no
// map bound, the constant environment radiance.
inline f3 sky(const orc_scene* s, f3 dir) {
    if (!s->hdri) return load3(s->sky);
    float u = atan2f(-dir.z, dir.x) * (float)(0.5 / 3.1415926) + 0.5f;
    float v = acosf(fmaxf(fminf(dir.y, 1.0f), -1.0f)) * (float)(1.0 / 3.1415926);
    const int W = s->hdri_w, H = s->hdri_h;
    float px = u * (float)W - 0.5f, py = v * (float)H - 0.5f;
    int ix = (int)std::floor(px), iy = (int)std::floor(py);
    float wx = px - (float)ix, wy = py - (float)iy;
    auto wrap = [](int a, int n) { a %= n; return a < 0 ? a + n : a; };
    auto F = [&](int a, int b) {
        const float* t = s->hdri + 4 * ((size_t)wrap(b, H) * W + wrap(a, W));
        return f3{t[0], t[1], t[2]};
    };
    auto L = [](f3 a, f3 b, float w) { return f3{lerpf(a.x, b.x, w), lerpf(a.y, b.y, w), lerpf(a.z, b.z, w)}; };
    f3 c = L(L(F(ix, iy), F(ix + 1, iy), wx), L(F(ix, iy + 1), F(ix + 1, iy + 1), wx), wy);
    return c * s->env_exp;
}

// ---------------------------------------------------------------------------
// DeterminateEstimatedHit(float& alpha, ...), core/render.cuh:105-197
// ---------------------------------------------------------------------------
bool estimated_hit(const orc_scene* s, float alpha, f3 pos, f3 dir, float dis, f3* next) {
    float smax = s->max_density * alpha;
    float t = 0, last_non_empty_t = 0, prob = 1.0f, last_dens = 0;
    float t_step = 2.0f / (float)s->res;
    float pass_rate = std::exp(-t_step * smax);
    float empty_step = 1.0f / (float)s->res;
    int loop = 0;
    while (loop++ < 10000) {
        if (t > dis) {
            if (last_non_empty_t != 0) { t = last_non_empty_t; break; }
            *next = {0, 0, 0};
            return false;
        }
        float d = density(s, pos + dir * t);
        if (d > 0) {
            float S = d * alpha;
            float step_p = pass_rate + (1.0f - pass_rate) * (1.0f - S / smax);
            float next_p = prob * step_p;
            if (next_p < 0.5f) {
                float offset = 1.0f - std::log(0.5f / prob) / std::log(step_p);
                t -= t_step * offset;
                break;
            }
            prob = next_p;
            t += t_step;
        } else {
            if (last_dens > 0) {
                float S = last_dens * alpha;
                float ts = t_step + d;
                float pr = std::exp(-(ts * smax));
                float step_p = pr + (1.0f - pr) * (1.0f - S / smax);
                float next_p = prob * step_p;
                if (next_p < 0.5f) {
                    float offset = 1.0f - std::log(0.5f / prob) / std::log(step_p);
                    t -= ts * offset;
                    break;
                }
                prob = next_p;
                last_non_empty_t = t + d;
            }
            t += fmax_(-d * 1.0f, empty_step);
        }
        last_dens = d;
    }
    *next = (dir * t) + pos;
    return true;
}

// GetMatrixFromNormal, core/render.cuh:694-708
void basis(f3 v1, float spread, Stream& st, f3 out[3]) {
    v1 = normalize(v1);
    f3 v2, v3;
    for (int guard = 0; guard < 1000; ++guard) {
        float ex = st.next() * spread;   // braced init: left to right
        float ey = st.next() * spread;
        f3 r = uniform_sphere(ex, ey);
        if (std::fabs(dot(r, v1)) < 0.00001) continue;
        v2 = normalize(cross(v1, r));
        v3 = cross(v2, v1);
        break;
    }
    out[0] = v1; out[1] = v2; out[2] = v3;
}

// MipTr / ShadowTerm_TRTex, core/renderResources.cu:229-272 (clamp addressing)
float shadow_tr(const orc_scene* s, f3 ori, f3 light, int mip) {
    const float* g = tr_ptr(s->tr_mips, mip);
    int n = 128 >> mip;
    if (ori.x < -0.5 || ori.y < -0.5 || ori.z < -0.5 || ori.x > 0.5 || ori.y > 0.5 || ori.z > 0.5) {
        float off = ray_box_offset(ori, light);
        if (off >= 0) return 1.0f * tex3(g, n, ori + light * off, true);
        return 1.0f;
    }
    return 1.0f * tex3(g, n, ori, true);
}

// SetupInputData, core/radiancePredict.cu:427-485
void setup_input(const orc_scene* s, bool active, f3 pos, f3 X, f3 Y, f3 Z, f3 LX, f3 L, float g,
                 float alpha, float* fv, float* fs, float* fh, float* gamma_out) {
    const float* dirs = T("STENCIL_DIRS");
    if (active) {
        int rand_index = 0;
        for (int i = 0; i < 192; ++i) {
            StencilEntry e = stencil(i);
            e.layer += 0.1f;
            int layer = (int)e.layer;
            f3 cur;
            if (e.type >= 4) {
                f3 p = load3(dirs + 3 * rand_index);
                cur = pos + ((X * p.x + Y * p.y + Z * p.z) * e.offset);
                rand_index++;
            } else {
                cur = pos + L * e.offset;
            }
            float d = tex3(mip_ptr(s->mips, layer), 256 >> layer, cur, false);
            fv[i] = std::log(1.0f + alpha * d / 64.0f);
            if (e.localindex == 0) {
                fh[i] = std::log(hg(dot(X, L), g) + 1.0f);
            } else {
                f3 ms = normalize(cur - pos);
                float radius = (float)(1 << layer) / 256.0f;
                float angle = std::atan(0.5f * radius / e.offset);
                float c1 = dot(X, ms), c2 = dot(LX, ms);
                float u = c1 * 0.5f + 0.5f, u2 = c2 * 0.5f + 0.5f;
                float v = angle / (3.1415926535f * 60.0f / 180.0f);
                float h0 = tex_lut(s->hg_lut, u, v), h1 = tex_lut(s->hg_lut, u2, v);
                fh[i] = std::log(h0 * h1 + 1.0f);
            }
            fs[i] = shadow_tr(s, cur, LX, std::max(layer - 1, 0));
        }
    } else {
        for (int i = 0; i < 192; ++i) fv[i] = fs[i] = fh[i] = 0;
    }
    float dd = dot(X, LX);
    dd = std::fmin(1.0f, std::fmax(-1.0f, dd));
    *gamma_out = std::acos(dd);
}

// DeterminateNextVertex, core/render.cuh:399-434.  The reference passes
// SampleHenyeyGreenstein(Rand(seed), Rand(seed), ...): argument order is
// unspecified in C++; the build fixes the x86-64 g++ order (right to left),
// i.e. the first draw is e1 and the second is e0.
bool next_vertex(const orc_scene* s, Stream& st, float alpha, float g, f3 pos, f3 dir, float dis,
                 f3* npos, f3* ndir) {
    float smax = s->max_density * alpha;
    float t = 0;
    int loop = 0;
    while (loop++ < 10000) {
        float rk = st.next();
        t -= std::log(1 - rk) / smax;
        if (t > dis) { *npos = {0, 0, 0}; *ndir = {0, 0, 0}; return false; }
        rk = st.next();
        float d = density(s, pos + dir * t);
        float S = d * alpha;
        if (S / smax > rk) break;
        if (d < 0) t -= d;
    }
    float e1 = st.next();
    float e0 = st.next();
    *ndir = sample_hg(e0, e1, dir, g);
    *npos = (dir * t) + pos;
    return true;
}

// Tr, core/render.cuh:60-103 (ratio tracking, then delta tracking)
float transmittance(const orc_scene* s, Stream& st, f3 pos, f3 dir, float dis, float alpha) {
    float smax = s->max_density * alpha;
    float tr = 1, t = 0;
    int loop = 0;
    while (loop++ < 10000 && tr > 0.5) {
        float rk = st.next();
        t -= std::log(1 - rk) / smax * s->tr_scale;
        if (t > dis) break;
        float d = density(s, pos + (dir * t));
        float S = d * alpha;
        tr *= 1 - fmax_(0.0f, S / smax);
        if (d < 0) t -= d;
    }
    while (loop++ < 10000 && tr > 0.001) {
        float rk = st.next();
        t -= std::log(1 - rk) / smax * s->tr_scale;
        if (t > dis) break;
        float d = density(s, pos + (dir * t));
        float S = d * alpha;
        if (st.next() < fmax_(0.0f, S / smax)) { tr = 0; break; }
        if (d < 0) t -= d;
    }
    return tr;
}

// fBm value-noise generator for the synthetic benchmark volumes.  Lattice hash:
// PCG-RXS-M-XS 32 (Jarzynski & Olano, "Hash Functions for GPU Rendering",
// JCGT 2020).  Interpolation: quintic smoothstep.  Not part of the reference.
inline uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
inline float lattice(uint32_t seed, int ix, int iy, int iz) {
    uint32_t h = pcg(pcg(pcg(pcg(seed) + (uint32_t)ix) + (uint32_t)iy) + (uint32_t)iz);
    return (float)(h >> 8) * 5.9604644775390625e-8f;
}
inline float quintic(float f) { return f * f * f * (f * (f * 6.0f - 15.0f) + 10.0f); }
float value_noise(float px, float py, float pz, uint32_t seed) {
    float fx = std::floor(px), fy = std::floor(py), fz = std::floor(pz);
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    float wx = quintic(px - fx), wy = quintic(py - fy), wz = quintic(pz - fz);
    float c00 = lerpf(lattice(seed, ix, iy, iz), lattice(seed, ix, iy, iz + 1), wz);
    float c01 = lerpf(lattice(seed, ix, iy + 1, iz), lattice(seed, ix, iy + 1, iz + 1), wz);
    float c10 = lerpf(lattice(seed, ix + 1, iy, iz), lattice(seed, ix + 1, iy, iz + 1), wz);
    float c11 = lerpf(lattice(seed, ix + 1, iy + 1, iz), lattice(seed, ix + 1, iy + 1, iz + 1), wz);
    return lerpf(lerpf(c00, c01, wy), lerpf(c10, c11, wy), wx);
}

}  // namespace

// ===========================================================================
// C API
// ===========================================================================
extern "C" {

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox(ctr, key, out); }

float orc_stream_uniform(uint32_t kind, uint32_t id, uint32_t sub, uint32_t frame, uint32_t seed, uint32_t n) {
    Stream st(kind, id, sub, frame, seed);
    float v = 0;
    for (uint32_t i = 0; i <= n; ++i) v = st.next();
    return v;
}

int orc_load_model(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return 1;
    char magic[8];
    uint32_t count = 0;
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "MRPNNMD1", 8) != 0 ||
        std::fread(&count, 4, 1, f) != 1) { std::fclose(f); return 2; }
    g_model.clear();
    for (uint32_t k = 0; k < count; ++k) {
        uint16_t len = 0;
        uint32_t n = 0;
        if (std::fread(&len, 2, 1, f) != 1) { std::fclose(f); return 3; }
        std::string name(len, '\0');
        if (std::fread(&name[0], 1, len, f) != len || std::fread(&n, 4, 1, f) != 1) { std::fclose(f); return 3; }
        std::vector<float> v(n);
        if (std::fread(v.data(), 4, n, f) != n) { std::fclose(f); return 3; }
        g_model[name] = std::move(v);
    }
    std::fclose(f);
    return 0;
}

int orc_model_tensor(const char* name, const float** data, int* count) {
    auto it = g_model.find(name);
    if (it == g_model.end()) return 1;
    *data = it->second.data();
    *count = (int)it->second.size();
    return 0;
}

float orc_fbm_voxel(int R, int x, int y, int z, uint32_t seed, float base_freq, int octaves, float gain) {
    float u = ((float)x + 0.5f) / (float)R, v = ((float)y + 0.5f) / (float)R, w = ((float)z + 0.5f) / (float)R;
    float sum = 0, norm = 0, amp = 1.0f, freq = base_freq;
    for (int o = 0; o < octaves; ++o) {
        sum = sum + amp * value_noise(u * freq, v * freq, w * freq, seed + (uint32_t)o * 1013u);
        norm = norm + amp;
        amp = amp * gain;
        freq = freq * 2.0f;
    }
    float n = sum / norm;
    float dx = u - 0.5f, dy = v - 0.5f, dz = w - 0.5f;
    float d = std::sqrt(dx * dx + dy * dy + dz * dz);
    // smoothstep(0.4, 0.32, d): 1 inside radius 0.32, 0 beyond 0.4
    float t = (d - 0.4f) / (0.32f - 0.4f);
    t = std::fmin(std::fmax(t, 0.0f), 1.0f);
    float fall = t * t * (3.0f - 2.0f * t);
    return std::fmin(std::fmax(n * fall, 0.0f), 1.0f);
}

void orc_fbm_volume(float* out, int R, uint32_t seed, float base_freq, int octaves, float gain) {
#pragma omp parallel for schedule(static)
    for (int x = 0; x < R; ++x)
        for (int y = 0; y < R; ++y)
            for (int z = 0; z < R; ++z)
                out[((size_t)x * R + y) * R + z] = orc_fbm_voxel(R, x, y, z, seed, base_freq, octaves, gain);
}

float orc_max_density(const float* d, int64_t n) {
    float m = 0.00001f;   // the reference's default max_density (core/volume.hpp:104)
    for (int64_t i = 0; i < n; ++i) m = std::fmax(m, d[i]);
    return m;
}

// VolumeRender::Update mip chain, core/volume.cu:1474-1515, with the CPU
// trilinear Sample() (border zero, negative clamp) of core/volume.cu:835-863
// and ParallelFill's texel centres (core/omp.cpp:4-18).
static float cpu_sample(const float* data, int res, float u, float v, float w) {
    f3 pos = subs(f3{u, v, w} * (float)res, 0.5f);
    int x = (int)std::floor(pos.x), y = (int)std::floor(pos.y), z = (int)std::floor(pos.z);
    f3 wt = pos - f3{(float)x, (float)y, (float)z};
    auto S = [&](int a, int b, int c) -> float {
        if (a < 0 || b < 0 || c < 0 || a >= res || b >= res || c >= res) return 0;
        return std::fmax(0.0f, data[((size_t)a * res + b) * res + c]);
    };
    return lerpf(lerpf(lerpf(S(x, y, z), S(x, y, z + 1), wt.z), lerpf(S(x, y + 1, z), S(x, y + 1, z + 1), wt.z), wt.y),
                 lerpf(lerpf(S(x + 1, y, z), S(x + 1, y, z + 1), wt.z), lerpf(S(x + 1, y + 1, z), S(x + 1, y + 1, z + 1), wt.z), wt.y),
                 wt.x);
}
static void fill_level(float* out, int res, const float* src, int src_res) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < res; ++i)
        for (int j = 0; j < res; ++j)
            for (int k = 0; k < res; ++k) {
                float u = (float)((i + 0.5) / res), v = (float)((j + 0.5) / res), w = (float)((k + 0.5) / res);
                out[((size_t)i * res + j) * res + k] = cpu_sample(src, src_res, u, v, w);
            }
}
void orc_build_pyramid(const float* data, int R, float* mips_out) {
    int res = 256;
    while (res * 2 < R) res <<= 1;
    const float* src = data;
    int src_res = R;
    std::vector<float> a, b;
    for (; res > 256; res >>= 1) {
        std::vector<float>& dst = (src == a.data()) ? b : a;
        dst.assign((size_t)res * res * res, 0.0f);
        fill_level(dst.data(), res, src, src_res);
        src = dst.data();
        src_res = res;
    }
    float* out = mips_out;
    for (int m = 0; m < 9; ++m) {
        int r = 256 >> m;
        fill_level(out, r, src, src_res);
        src = out;
        src_res = r;
        out += (size_t)r * r * r;
    }
}

// Fill_TR, core/volume.cu:1535-1560, bound to mips[level+1] with alpha scaled
// by 1.73^(level+1) (core/volume.cu:1636-1653).
void orc_tr_mip_level(const float* mips, int level, float alpha, const float light_dir[3], float* out) {
    int res = 128 >> level;
    const float* src = mip_ptr(mips, level + 1);
    float a = alpha / std::pow(1.73f, (float)level + 1.0f);
    f3 L = load3(light_dir);
#pragma omp parallel for schedule(dynamic, 1)
    for (int x = 0; x < res; ++x)
        for (int y = 0; y < res; ++y)
            for (int z = 0; z < res; ++z) {
                f3 uv = adds(f3{(float)x, (float)y, (float)z}, 0.5f) / (float)res;
                f3 ori = subs(uv, 0.5f);
                float dis = ray_box_distance(ori, L);
                float inv_step = dis / 128;
                f3 lp = ori;
                float acc = 0;
                for (int i = 0; i < 128; ++i) {
                    lp = lp + L * inv_step;
                    acc = acc + tex3(src, res, lp, false);
                }
                out[((size_t)x * res + y) * res + z] = 1.0f * (std::exp(-acc * a * inv_step) * 1.0f);
            }
}

// Scrambled radical inverse (core/volume.cu:1186-1319 restates PBRT's
// ScrambledRadicalInverse) with the reference's digit permutations for bases
// 2-11 (RadicalInversePermutations_, core/volume.cu:1195), which the model
// file carries as HALTON_PERMS; bn is a per-texel Philox draw instead of a
// curand draw (the reference's draw depends on curand's XORWOW state, which
// no other generator reproduces).
namespace {
const uint32_t kPrimes[5] = {2, 3, 5, 7, 11};
const uint32_t kPrimeSums[5] = {0, 2, 5, 10, 17};
uint32_t g_perm[28];
void make_perms() {   // from the loaded model, before each table build
    const float* p = T("HALTON_PERMS");
    for (int i = 0; i < 28; ++i) g_perm[i] = (uint32_t)p[i];
}
float scrambled_radical_inverse(uint32_t bi, uint32_t a) {
    const uint32_t base = kPrimes[bi], off = kPrimeSums[bi];
    const float inv_base = (float)1 / (float)base;
    uint32_t rev = 0;
    float inv_base_n = 1;
    while (a) {
        uint32_t next = a / base;
        uint32_t digit = a - next * base;
        rev = rev * base + g_perm[off + digit];
        inv_base_n *= inv_base;
        a = next;
    }
    return fmin_(inv_base_n * ((float)rev + inv_base * (float)g_perm[off] / (1 - inv_base)), 0.99999994f);
}
inline float fracf(float f) { return f - (float)(long)f; }   // vector.cu:20
}  // namespace

// Fill_Hg, core/volume.cu:1322-1400, for a list of texels (index j*512+i).
void orc_hg_lut_texels(float g, uint32_t seed, const int* texels, int n, float* out) {
    make_perms();
#pragma omp parallel for schedule(dynamic, 64)
    for (int q = 0; q < n; ++q) {
        int i = texels[q] % LUT, j = texels[q] / LUT;
        float costheta = (float)((((float)i + 0.5) / LUT) * 2.0 - 1.0);
        float aa = (float)(((float)j + 0.5) / LUT);
        float angle = (float)(aa * 3.1415926535 * 60.0 / 180.0);
        Stream st(1, (uint32_t)texels[q], 0, 0, seed);
        float bn = st.next();
        float h = 0.0f;
        float radius = std::tan(angle);
        f3 view = {1.0f, 0.0f, 0.0f};
        f3 dir = {costheta, std::sqrt(1.0f - costheta * costheta), 0.0f};
        float mis = 0;
        {
            float p = radius * radius - 1 + dir.x * dir.x;
            if (p > 0) {
                float sdotl = g > 0 ? dir.x : -dir.x;
                float w = std::sqrt(p);
                float d0 = fmax_(0.0f, sdotl - w) / radius;
                float d1 = (sdotl + w) / radius;
                float d = d1 * d1 * d1 - d0 * d0 * d0;
                mis = (float)(d1 > d0) * d;
            }
            mis = fmin_(fmax_(mis, 1e-8f), 1.0f);
            float a = std::fabs(g);
            a = (float)(a < 0.6 ? 0 : (a < 0.7 ? (a - 0.6) * 9 : (std::pow((a - 0.7) / 0.3, 0.05) * 0.1 + 0.9)));
            mis = 1 - 1 / (1 + a * mis / (1 - a));
        }
        for (uint32_t k = 0; k < 1024; ++k) {
            if (fracf(scrambled_radical_inverse(4, k) + bn) < mis) {
                float rx = fracf(scrambled_radical_inverse(0, k) + bn);
                float ry = fracf(scrambled_radical_inverse(1, k) + bn);
                f3 l = sample_hg(rx, ry, view, g);
                float sdotl = dot(dir, l);
                float p = radius * radius - 1 + sdotl * sdotl;
                if (p <= 0) continue;
                float w = std::sqrt(p);
                float d0 = sdotl - w;
                float d1 = (sdotl + w) / radius;
                d0 = fmax_(0.0f, d0) / radius;
                float d = d1 * d1 * d1 - d0 * d0 * d0;
                h += fmax_(0.0f, d / 4);
            } else {
                float rx = fracf(scrambled_radical_inverse(0, k) + bn);
                float ry = fracf(scrambled_radical_inverse(1, k) + bn);
                float rz = fracf(scrambled_radical_inverse(2, k) + bn);
                float theta = (float)(rx * 2.0 * 3.1415926535);
                float phi = (float)std::acos(2.0 * ry - 1.0);
                float r = std::pow(rz, 1 / 3.0f);
                float st_ = std::sin(theta), ct = std::cos(theta), sp = std::sin(phi), cp = std::cos(phi);
                float x = radius * r * sp * ct, y = radius * r * sp * st_, z = radius * r * cp;
                f3 rp = f3{x, y, z} + dir;
                float c = dot(normalize(rp), view);
                h += hg(c, g);
            }
        }
        h /= 1024;
        out[q] = h;
    }
}

// Fill_BakeTR, core/volume.cu:1562-1587.  With replicate_reference_seeding
// the stream restarts for each of the sampCount estimates, as InitRand inside
// the loop does in the reference (the estimates are then identical).
void orc_baked_tr(const orc_scene* s, float alpha, const float light_dir[3], int bake_res, uint32_t seed,
                  int replicate_reference_seeding, const int64_t* voxels, int64_t n, float* out) {
    f3 L = load3(light_dir);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t q = 0; q < n; ++q) {
        int64_t vi = voxels[q];
        int x = (int)(vi / ((int64_t)bake_res * bake_res)), y = (int)((vi / bake_res) % bake_res), z = (int)(vi % bake_res);
        f3 uv = adds(f3{(float)x, (float)y, (float)z}, 0.5f) / (float)bake_res;
        f3 p = subs(uv, 0.5f);
        int cnt = (density(s, p) > 0) ? 5 : 2;
        float acc = 0;
        for (int i = 0; i < cnt; ++i) {
            Stream st(2, (uint32_t)vi, replicate_reference_seeding ? (uint32_t)(vi >> 32) * 8u : (uint32_t)(vi >> 32) * 8u + (uint32_t)i, 0, seed);
            float md = ray_box_distance(p, L);
            acc += transmittance(s, st, p, L, md, alpha);
        }
        out[q] = 1.0f * (acc / cnt);
    }
}

float orc_tr(const orc_scene* s, const float pos[3], const float dir[3], float dis, float alpha, uint32_t stream_id,
             uint32_t sub, uint32_t frame, uint32_t seed, uint32_t kind) {
    Stream st(kind, stream_id, sub, frame, seed);
    return transmittance(s, st, load3(pos), load3(dir), dis, alpha);
}

void orc_stencil_tables(float* offset, int* layer, int* type, int* localindex, float* lut_v) {
    for (int i = 0; i < 192; ++i) {
        StencilEntry e = stencil(i);
        e.layer += 0.1f;
        int l = (int)e.layer;
        offset[i] = e.offset;
        layer[i] = l;
        type[i] = e.type;
        localindex[i] = e.localindex;
        float radius = (float)(1 << l) / 256.0f;
        float angle = std::atan(0.5f * radius / e.offset);
        lut_v[i] = angle / (3.1415926535f * 60.0f / 180.0f);
    }
}

float orc_hg(float c, float g) { return hg(c, g); }
void orc_sample_hg(float e0, float e1, const float v[3], float g, float out[3]) { store3(out, sample_hg(e0, e1, load3(v), g)); }
float orc_ray_box_offset(const float p[3], const float d[3]) { return ray_box_offset(load3(p), load3(d)); }
float orc_ray_box_distance(const float p[3], const float d[3]) { return ray_box_distance(load3(p), load3(d)); }
float orc_sample_density(const float* grid, int n, const float pos[3], int clamp_mode) {
    return tex3(grid, n, load3(pos), clamp_mode != 0);
}
float orc_sample_lut(const float* lut, float u, float v) { return tex_lut(lut, u, v); }

// RenderCamera ray, core/volume.cu:208-216
void orc_camera_ray(const orc_view* v, int row, int col, float dir_out[3]) {
    Stream st(0, (uint32_t)(row * v->width + col), 0, (uint32_t)v->frame, v->seed);
    float r0 = st.next(), r1 = st.next();
    float u = 1 - ((float)col + r0) / (float)v->width;
    float w = 1 - ((float)row + r1) / (float)v->height;
    f3 ori = load3(v->ori);
    f3 fwd = normalize(neg(ori));
    f3 d = fwd + (load3(v->right) * (u * 2 - 1)) + (load3(v->up) * (w * 2 - 1));
    store3(dir_out, normalize(d));
}

// GetSamplePoint, core/render.cuh:436-462
int orc_first_hit(const orc_scene* s, const float ori_[3], const float dir_[3], float alpha, float hit_out[3]) {
    f3 ori = load3(ori_), dir = normalize(load3(dir_));
    store3(hit_out, f3{0, 0, 0});
    float dis = ray_box_offset(ori, dir);
    if (dis < 0) return 0;
    f3 sp = ori + dir * dis;
    float md = ray_box_distance(sp, dir);
    f3 p;
    bool in = estimated_hit(s, alpha, sp, dir, md, &p);
    if (in) store3(hit_out, p);
    return in ? 1 : 0;
}

void orc_basis(const float v[3], float spread, uint32_t id, uint32_t sub, uint32_t frame, uint32_t seed,
               uint32_t* cursor, float out9[9]) {
    Stream st(0, id, sub, frame, seed);
    for (uint32_t i = 0; i < *cursor; ++i) st.next();
    f3 b[3];
    basis(load3(v), spread, st, b);
    *cursor = st.n;
    for (int k = 0; k < 3; ++k) store3(out9 + 3 * k, b[k]);
}

void orc_setup_input(const orc_scene* s, int active, const float pos[3], const float X[3], const float Y[3],
                     const float Z[3], const float LX[3], const float light[3], float g, float alpha,
                     float* feat576, float* gamma_out) {
    setup_input(s, active != 0, load3(pos), load3(X), load3(Y), load3(Z), load3(LX), load3(light), g, alpha,
                feat576, feat576 + 192, feat576 + 384, gamma_out);
}

void orc_mlp_f32(const float* feat, const float* gamma, float g, const float sr[3], int n, float* out3) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
        float o[3];
        mlp_one<float>(feat + (size_t)i * 576, gamma[i], g, sr, o);
        out3[3 * i] = o[0]; out3[3 * i + 1] = o[1]; out3[3 * i + 2] = o[2];
    }
}
void orc_mlp_f64(const float* feat, const float* gamma, float g, const float sr[3], int n, double* out3) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
        double o[3];
        mlp_one<double>(feat + (size_t)i * 576, gamma[i], g, sr, o);
        out3[3 * i] = o[0]; out3[3 * i + 1] = o[1]; out3[3 * i + 2] = o[2];
    }
}

// RenderCamera<true, MRPNN> + NNPredict<MRPNN>, core/volume.cu:198-228 and
// core/render.cuh:808-875.  Output per pixel for one launch, after the
// max(0, .) clamp of RenderCamera; the running mean is the caller's.
void orc_predict_pixels(const orc_scene* s, const orc_view* v, const int* pixels, int n, float* rgba_out,
                        float* feat_out, float* gamma_out, float* hit_out) {
    f3 sr1 = load3(s->scatter_rate) / 1.001f;
    float sr[3] = {sr1.x, sr1.y, sr1.z};
#pragma omp parallel for schedule(dynamic, 8)
    for (int q = 0; q < n; ++q) {
        int pix = pixels[q];
        int row = pix / v->width, col = pix % v->width;
        float d0[3];
        orc_camera_ray(v, row, col, d0);
        f3 ori = load3(v->ori);
        f3 dir = normalize(load3(d0));
        f3 L = normalize(load3(v->light_dir));
        Stream st(0, (uint32_t)pix, 0, (uint32_t)v->frame, v->seed);   // InitRand again
        float hit[3];
        int active = orc_first_hit(s, v->ori, &dir.x, v->alpha, hit);
        f3 main_b[3], light_b[3];
        basis(dir, 0.1f, st, main_b);
        basis(L, 0.1f, st, light_b);
        float feat[576], gamma;
        setup_input(s, active != 0, load3(hit), main_b[0], main_b[1], main_b[2], light_b[0], L, v->g, v->alpha,
                    feat, feat + 192, feat + 384, &gamma);
        float o[4];
        if (active) {
            float p[3];
            mlp_one<float>(feat, gamma, v->g, sr, p);
            f3 pr = f3{p[0], p[1], p[2]} * 1.0f;   // alphaMult == 1
            f3 res = (pr * load3(v->light_color)) * load3(s->scatter_rate);
            o[0] = res.x; o[1] = res.y; o[2] = res.z;
            o[3] = length(ori - load3(hit));
        } else {
            f3 sk = sky(s, dir);
            o[0] = sk.x; o[1] = sk.y; o[2] = sk.z; o[3] = -1;
        }
        for (int c = 0; c < 4; ++c) rgba_out[4 * q + c] = fmax_(0.0f, o[c]);
        if (feat_out) std::memcpy(feat_out + (size_t)q * 576, feat, sizeof feat);
        if (gamma_out) gamma_out[q] = gamma;
        if (hit_out) { hit_out[4 * q] = hit[0]; hit_out[4 * q + 1] = hit[1]; hit_out[4 * q + 2] = hit[2]; hit_out[4 * q + 3] = (float)active; }
    }
}

// One sample of CalculateRadiance's loop (core/render.cuh:553-592) from the
// box entry ori + dir * dis; NEE through the baked grid, or one Tr()
// estimate per vertex from nst when the scene has no baked grid.
static f3 trace_sample(const orc_scene* s, const orc_view* v, f3 ori, f3 dir, float dis, f3 L, Stream& st,
                       Stream& nst) {
    f3 lc = load3(v->light_color);
    f3 srate = load3(s->scatter_rate);
    f3 res = {0, 0, 0};
    f3 p = ori + dir * dis, rd = dir, csr = {1, 1, 1};
    for (int b = 0; b < v->multi_scatter; ++b) {
        f3 np, nd;
        float md = ray_box_distance(p, rd);
        if (!next_vertex(s, st, v->alpha, v->g, p, rd, md, &np, &nd)) {
            res = res + sky(s, rd) * csr;
            break;
        }
        p = np;
        csr = csr * srate;
        float ph = hg(dot(rd, L), v->g);
        float tr = s->baked_tr ? tex3(s->baked_tr, s->baked_res, p, true)
                               : transmittance(s, nst, p, L, ray_box_distance(p, L), v->alpha);
        res = res + (lc * csr) * (tr * ph);
        rd = nd;
    }
    return res;
}

// RenderCamera<false> + CalculateRadiance, core/volume.cu:198-228 and
// core/render.cuh:535-597.  Sample k of a launch draws from its own stream
// (sub = k); the first sample restarts the pixel stream like InitRand does.
void orc_trace_pixels(const orc_scene* s, const orc_view* v, const int* pixels, int n, float* rgba_out,
                      double* sum3, double* sumsq3) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int q = 0; q < n; ++q) {
        int pix = pixels[q];
        int row = pix / v->width, col = pix % v->width;
        float d0[3];
        orc_camera_ray(v, row, col, d0);
        f3 ori = load3(v->ori);
        f3 dir = normalize(load3(d0));
        f3 L = normalize(load3(v->light_dir));
        float dis = ray_box_offset(ori, dir);
        double acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0};
        float out[4];
        if (dis < 0) {
            f3 sk = sky(s, dir);
            for (int c = 0; c < 3; ++c) { float x = (&sk.x)[c]; acc[c] = (double)x * v->spp; acc2[c] = (double)x * x * v->spp; }
            out[0] = sk.x; out[1] = sk.y; out[2] = sk.z; out[3] = -1;
        } else {
            float coverage = 0;
            bool any = false;
            for (int k = 0; k < v->spp; ++k) {
                Stream st(0, (uint32_t)pix, (uint32_t)k, (uint32_t)v->frame, v->seed);
                // unbiased NEE (no baked grid): one Tr() estimate per vertex
                // from the sample's own NEE stream (kind 3)
                Stream nst(3, (uint32_t)pix, (uint32_t)k, (uint32_t)v->frame, v->seed);
                f3 res = trace_sample(s, v, ori, dir, dis, L, st, nst);
                for (int c = 0; c < 3; ++c) { double x = (&res.x)[c]; acc[c] += x; acc2[c] += x * x; }
                // coverage: the reference tests its running sum (render.cuh:594)
                any = any || res.x > 0 || res.y > 0 || res.z > 0;
                coverage += any ? 1.0f : 0.0f;
            }
            for (int c = 0; c < 3; ++c) out[c] = (float)(acc[c] / v->spp);
            out[3] = coverage / (float)v->spp;
        }
        for (int c = 0; c < 4; ++c) rgba_out[4 * q + c] = fmax_(0.0f, out[c]);
        if (sum3) for (int c = 0; c < 3; ++c) { sum3[3 * q + c] = acc[c]; sumsq3[3 * q + c] = acc2[c]; }
    }
}


// GetRadiances with RenderType PT (core/volume.cu:405-479 ->
// CalculateRadianceMulti<0> -> CalculateRadiance) for explicit rays: ray q,
// sample k draws from stream (0, q, k, frame, seed).  FP64 sums per channel.
void orc_trace_rays(const orc_scene* s, const orc_view* v, const float* ori_, const float* dir_, int n, double* sum3,
                    double* sumsq3) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int q = 0; q < n; ++q) {
        f3 ori = load3(ori_ + 3 * q), dir = normalize(load3(dir_ + 3 * q));
        f3 L = normalize(load3(v->light_dir));
        float dis = ray_box_offset(ori, dir);
        double acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0};
        for (int k = 0; k < v->spp; ++k) {
            f3 res = sky(s, dir);
            if (dis >= 0) {
                Stream st(0, (uint32_t)q, (uint32_t)k, (uint32_t)v->frame, v->seed);
                Stream nst(3, (uint32_t)q, (uint32_t)k, (uint32_t)v->frame, v->seed);
                res = trace_sample(s, v, ori, dir, dis, L, st, nst);
            }
            for (int c = 0; c < 3; ++c) { double x = (&res.x)[c]; acc[c] += x; acc2[c] += x * x; }
        }
        for (int c = 0; c < 3; ++c) { sum3[3 * q + c] = acc[c]; sumsq3[3 * q + c] = acc2[c]; }
    }
}

// GetSample (core/render.cuh:615-655), the training-data generator: from a
// point in the medium, the first direction HG-sampled around dir, up to
// multi_scatter bounces, NEE by Tr() on the same stream.  Task q draws from
// one stream (4, q, 0, 0, seed) across its samples, as the reference's one
// InitRand per thread.
void orc_get_samples(const orc_scene* s, const float* alpha, const float* ori, const float* dir, const float* ldir,
                     const float* g, const float* scatter, int n, const float lc_[3], int multi_scatter, int spp,
                     uint32_t seed, float* out3) {
    f3 lc = load3(lc_);
#pragma omp parallel for schedule(dynamic, 4)
    for (int q = 0; q < n; ++q) {
        Stream st(4, (uint32_t)q, 0, 0, seed);
        f3 o = load3(ori + 3 * q), d = load3(dir + 3 * q), L = load3(ldir + 3 * q);
        float a = alpha[q], gq = g[q], sc = scatter[q];
        f3 res = {0, 0, 0};
        for (int i = 0; i < spp; ++i) {
            f3 pos = o;
            float e1 = st.next();
            float e0 = st.next();
            f3 rd = sample_hg(e0, e1, d, gq);
            f3 csr = {1, 1, 1};
            for (int b = 0; b < multi_scatter; ++b) {
                f3 np, nd;
                float dis = ray_box_distance(pos, rd);
                if (!next_vertex(s, st, a, gq, pos, rd, dis, &np, &nd)) {
                    res = res + sky(s, rd) * csr;
                    break;
                }
                pos = np;
                csr = (csr * 1.001f) * sc;
                dis = ray_box_distance(pos, L);
                float phase = hg(dot(rd, L), gq);
                res = res + (lc * csr) * (transmittance(s, st, pos, L, dis, a) * phase);
                rd = nd;
            }
        }
        store3(out3 + 3 * q, f3{res.x / (float)spp, res.y / (float)spp, res.z / (float)spp});
    }
}

// GetTrs -> ShadowTerm_TRs (core/render.cuh:668-680): light colour x pi x the
// mean of Tr() x HG over spp estimates; task q draws from stream (5, q, 0, 0, seed).
void orc_get_trs(const orc_scene* s, float alpha, const float* ori, const float* dir, int n, const float L_[3],
                 const float lc_[3], float g, int spp, uint32_t seed, float* out3) {
    f3 L = load3(L_), lc = load3(lc_);
#pragma omp parallel for schedule(dynamic, 16)
    for (int q = 0; q < n; ++q) {
        Stream st(5, (uint32_t)q, 0, 0, seed);
        f3 o = load3(ori + 3 * q), d = load3(dir + 3 * q);
        float res = 0;
        for (int i = 0; i < spp; ++i) {
            float dis = ray_box_distance(o, L);
            float phase = hg(dot(d, L), g);
            res = res + transmittance(s, st, o, L, dis, alpha) * phase;
        }
        f3 r = lc * 3.1415926535f;
        store3(out3 + 3 * q, f3{r.x * res / (float)spp, r.y * res / (float)spp, r.z * res / (float)spp});
    }
}

// ---------------------------------------------------------------------------
// Interactive frame (VolumeRender::Render(float3*, Histogram*, ...),
// core/volume.cu:57-196, 230-353, 550-628; tone maps core/render.cuh:1144-1236).
// Histogram layout: bin[30], total, x2, x (33 floats per pixel).
// ---------------------------------------------------------------------------
static f3 mat3(f3 r0, f3 r1, f3 r2, f3 v) { return f3{dot(r0, v), dot(r1, v), dot(r2, v)}; }
static f3 lerp3(f3 a, f3 b, float t) { return f3{lerpf(a.x, b.x, t), lerpf(a.y, b.y, t), lerpf(a.z, b.z, t)}; }
static f3 gamma_tone(f3 c) {
    float e = 1.0f / 2.2f;
    return f3{std::pow(c.x, e), std::pow(c.y, e), std::pow(c.z, e)};
}
static f3 aces_tone(f3 color) {
    const f3 A0 = {0.6624541811f, 0.1340042065f, 0.1561876870f}, A1 = {0.2722287168f, 0.6740817658f, 0.0536895174f},
             A2 = {-0.0055746495f, 0.0040607335f, 1.0103391003f};
    f3 aces = mat3({0.4397010f, 0.3829780f, 0.1773350f}, {0.0897923f, 0.8134230f, 0.0967616f},
                   {0.0175440f, 0.1115440f, 0.8707040f}, color);
    const f3 Y = {0.272229f, 0.674082f, 0.0536895f};
    f3 cg = mat3({1.4514393161f, -0.2365107469f, -0.2149285693f}, {-0.0765537734f, 1.1762296998f, -0.0996759264f},
                 {0.0083161484f, -0.0060324498f, 0.9977163014f}, aces);
    float tmp = dot(cg, Y);
    cg = lerp3(f3{tmp, tmp, tmp}, cg, 0.96f);
    const float a = 278.5085f, b = 10.7772f, c = 293.6045f, d = 88.7122f, e = 80.6889f;
    f3 x = cg;
    f3 num = x * ((x * a) + f3{b, b, b});
    f3 den = (x * ((x * c) + f3{d, d, d})) + f3{e, e, e};
    f3 post = {num.x / den.x, num.y / den.y, num.z / den.z};
    f3 XYZ = mat3(A0, A1, A2, post);
    float divisor = fmax_(dot(XYZ, f3{1, 1, 1}), 1e-4f);
    f3 xyY = {XYZ.x / divisor, XYZ.y / divisor, XYZ.y};
    xyY.z = fmin_(fmax_(xyY.z, 0.0f), 65504.0f);
    xyY.z = std::pow(xyY.z, 0.9811f);
    float m = xyY.z / fmax_(xyY.y, 1e-4f);
    XYZ = f3{xyY.x * m, xyY.z, ((1.0f - xyY.x) - xyY.y) * m};
    f3 lin = mat3({1.6410233797f, -0.3248032942f, -0.2364246952f}, {-0.6636628587f, 1.6153315917f, 0.0167563477f},
                  {0.0117218943f, -0.0082844420f, 0.9883948585f}, XYZ);
    tmp = dot(lin, Y);
    lin = lerp3(f3{tmp, tmp, tmp}, lin, 0.93f);
    XYZ = mat3(A0, A1, A2, lin);
    XYZ = mat3({0.98722400f, -0.00611327f, 0.0159533f}, {-0.00759836f, 1.00186000f, 0.0053302f},
               {0.00307257f, -0.00509595f, 1.0816800f}, XYZ);
    lin = mat3({3.2409699419f, -1.5373831776f, -0.4986107603f}, {-0.9692436363f, 1.8759675015f, 0.0415550574f},
               {0.0556300797f, -0.2039769589f, 1.0569715142f}, XYZ);
    return gamma_tone(lin);
}
static float saturate1(float v) { return fmin_(fmax_(v, 0.0f), 1.0f); }
static int unroll(int row, int col, int W, int H) {
    col = std::min(std::max(0, col), W - 1);
    row = std::min(std::max(0, row), H - 1);
    return col + W * row;
}
static float compare_histo(const float* x, const float* y) {
    float nx = x[30], ny = y[30];
    float sy = std::sqrt(ny / nx), sx = std::sqrt(nx / ny);
    float p = 0, res = 0;
    for (int i = 0; i < 30; ++i) {
        float hx = x[i], hy = y[i];
        if (hx != 0 || hy != 0) {
            p += 1;
            float t = sy * hx - sx * hy;
            res += t * t / (hx + hy);
        }
    }
    return p == 0 ? 0 : res / p;
}

void orc_frame_pt(const orc_scene* s, const orc_view* v, int fnum, int checker, int flip, float* target,
                  float* histo) {
    const int W = v->width, H = v->height;
#pragma omp parallel for schedule(dynamic, 16)
    for (int idx = 0; idx < W * H; ++idx) {
        int row = idx / W, col = idx % W;
        if (checker && ((row + col + flip) & 1)) continue;
        Stream st(0, (uint32_t)idx, 0, (uint32_t)v->frame, v->seed);
        float r0 = st.next(), r1 = st.next();
        float u = 1 - ((float)col + r0) / (float)W;
        float w = ((float)row + r1) / (float)H;
        f3 ori = load3(v->ori);
        f3 fwd = normalize(neg(ori));
        f3 dir = normalize(fwd + (load3(v->right) * (u * 2 - 1)) + (load3(v->up) * (w * 2 - 1)));
        dir = normalize(dir);   // CalculateRadiance normalizes its direction again (core/render.cuh:540)
        f3 L = normalize(load3(v->light_dir));
        float dis = ray_box_offset(ori, dir);
        f3 res = sky(s, dir);
        if (dis >= 0) {
            Stream s0(0, (uint32_t)idx, 0, (uint32_t)v->frame, v->seed);
            Stream nst(3, (uint32_t)idx, 0, (uint32_t)v->frame, v->seed);
            res = trace_sample(s, v, ori, dir, dis, L, s0, nst);
        }
        res = f3{fmax_(0.0f, res.x), fmax_(0.0f, res.y), fmax_(0.0f, res.z)};
        float* h = histo + 33 * (size_t)idx;
        if (fnum == 0) for (int k = 0; k < 33; ++k) h[k] = 0;
        float rate = 1.0f / (float)(1 + fnum);
        f3 t = lerp3(load3(target + 3 * (size_t)idx), res, rate);
        store3(target + 3 * (size_t)idx, t);
        res = f3{res.x / (res.x + 1), res.y / (res.y + 1), res.z / (res.z + 1)};
        h[30] += 1;
        int bx = (int)std::floor(fmin_(res.x, 0.999f) * 10.0f), by = (int)std::floor(fmin_(res.y, 0.999f) * 10.0f),
            bz = (int)std::floor(fmin_(res.z, 0.999f) * 10.0f);
        h[bx] += 1;
        h[by + 10] += 1;
        h[bz + 20] += 1;
        float l = dot(res, f3{1, 1, 1});
        h[32] = lerpf(h[32], l, rate);
        h[31] = lerpf(h[31], l * l, rate);
    }
}

void orc_frame_finish(const float* target, float* histo, int W, int H, int frame_num, int flip, int predict,
                      int denoise, float exposure, int tone, uint32_t* rgba8) {
#pragma omp parallel for schedule(static)
    for (int id = 0; id < W * H; ++id) {
        int row = id / W, col = id % W;
        auto T = [&](int i) { return load3(target + 3 * (size_t)i); };
        f3 res;
        if (predict) {
            res = T(id);
        } else if (frame_num == 0) {
            if ((((row + flip) % 2) + col) % 2 == 0) {
                res = T(id);
            } else {
                res = ((T(unroll(row - 1, col, W, H)) + T(unroll(row + 1, col, W, H))) + T(unroll(row, col - 1, W, H))) +
                      T(unroll(row, col + 1, W, H));
                res = f3{res.x / 4.0f, res.y / 4.0f, res.z / 4.0f};
            }
        } else {
            const float* c = histo + 33 * (size_t)id;
            float variance = std::fabs(c[31] - c[32] * c[32]);
            if (denoise && variance > 0.01) {
                res = f3{0, 0, 0};
                float ws = 0;
                for (int i = -5; i <= 5; ++i)
                    for (int j = -5; j <= 5; ++j) {
                        int t = unroll(row + i, col + j, W, H);
                        float w = (float)std::fmax(0.0, 1.0 - 1.2 * (double)compare_histo(c, histo + 33 * (size_t)t));
                        res = res + T(t) * w;
                        ws += w;
                    }
                res = f3{res.x / ws, res.y / ws, res.z / ws};
            } else {
                res = T(id);
            }
        }
        f3 val = res * exposure;
        if (tone == 1) val = gamma_tone(val);
        else if (tone == 2) val = aces_tone(val);
        uint32_t r = (uint32_t)(255.0f * saturate1(val.x)), g = (uint32_t)(255.0f * saturate1(val.y)),
                 b = (uint32_t)(255.0f * saturate1(val.z));
        rgba8[id] = 0xff000000u | (r << 16) | (g << 8) | b;
    }
    if (predict)
        for (int id = 0; id < W * H; ++id) {
            f3 t = load3(target + 3 * (size_t)id);
            histo[33 * (size_t)id + 30] = t.x;
            histo[33 * (size_t)id + 32] = t.y;
            histo[33 * (size_t)id + 31] = t.z;
        }
}

// ---------------------------------------------------------------------------
// Tile gather of the tile network (GatherData -> GatherSamples ->
// NNGatherSamples, core/volume.cu:257-282, 630-700; core/render.cuh:298-397,
// 464-485, 1006-1142; SetupInputData2, core/radiancePredict.cu:487-553).
// 773 floats per tile: X_Val[192], X_Val_Hg[192], X_Val_Sub[192], 5 angle /
// depth-gradient terms, 192 t-grid values.  neg_logs = {-log 0.76, -log 0.75,
// -log 0.25} (host logf, as the reference computes them in the loop).
// ---------------------------------------------------------------------------
static bool check_exit(float S, float lastS, float dt, float t, float& tau, float& tau_target, float ts[4],
                       bool& first_hit, float tau_second) {
    float tau_next = tau + (S + lastS) * 0.5f * dt;
    if (tau_next >= tau_target) {
        float dtau = tau_target - tau;
        float A = 0.5f * dt * (S - lastS), B = dt * lastS, C = -dtau;
        auto solve = [&](float Cq, float dq) {
            float off;
            if (std::fabs(A) < 1e-6f) {
                off = dq / (dt * (S + lastS) * 0.5f);
            } else {
                float D = B * B - 4.0f * A * Cq;
                D = fmax_(D, 0.0f);
                float sq = std::sqrt(D);
                float q = (float)(-0.5 * (double)(B + sq));
                float u1 = q / A, u2 = Cq / q;
                off = (u1 == fmin_(fmax_(u1, 0.0f), 1.0f)) ? u1 : u2;
            }
            return off;
        };
        float off = solve(C, dtau);
        off = fmin_(fmax_(off, 0.0f), 1.0f);
        float hit_t = t - dt * (1.0f - off);
        if (first_hit) {
            ts[0] = hit_t;
            tau_target = tau_second;
            first_hit = false;
            if (tau_next >= tau_target) {
                float d2 = tau_target - tau;
                float off2 = solve(-d2, d2);
                ts[1] = t - dt * (1.0f - off2);
                return true;
            }
        } else {
            ts[1] = hit_t;
            return true;
        }
    }
    tau = tau_next;
    return false;
}

static void estimated_hit_ts(const orc_scene* s, float alpha, f3 pos, f3 dir, float dis, const float nl[3],
                             float ts[4]) {
    float smax = s->max_density * alpha;
    float t = 0;
    ts[0] = 0; ts[1] = 0; ts[2] = FLT_MAX; ts[3] = 0;
    float last_non_empty_t = 0;
    float t_step = 1.0f / (float)s->res;
    if (smax * t_step > nl[0]) t_step = nl[0] / smax;
    float tau = 0, tau_target = nl[1];
    bool first = true;
    int loop = 0;
    float last = 0;
    while (loop++ < 10000) {
        if (t > dis) {
            if (first) ts[0] = last_non_empty_t;
            else ts[1] = last_non_empty_t;
            break;
        }
        float d = density(s, pos + dir * t);
        if (d > 0) {
            float S = d * alpha;
            if (check_exit(S, last, t_step, t, tau, tau_target, ts, first, nl[2])) break;
            ts[2] = fmin_(t, ts[2]);
            t += t_step;
            last = S;
        } else {
            if (last > 0) {
                float ts_ = t_step + d;
                if (ts_ > 0) {
                    if (check_exit(0.0f, last, ts_, t, tau, tau_target, ts, first, nl[2])) break;
                    last_non_empty_t = t + ts_;
                } else {
                    last_non_empty_t = t;
                }
            }
            t += fmax_(-d * 1.0f, 0.5f / (float)s->res);
            last = 0.0f;
        }
    }
    if (ts[2] == FLT_MAX) ts[2] = 0.0f;
    float survival = std::exp(-tau);
    ts[3] = fmin_(fmax_(1.0f - survival, 0.0f) / 0.75f, 1.0f);
}

static void sample_t(const orc_scene* s, f3 ori, f3 dir, float alpha, const float nl[3], float ts[4]) {
    float dis = ray_box_offset(ori, dir);
    if (dis < 0) { ts[0] = ts[1] = ts[2] = ts[3] = 0; return; }
    f3 sp = ori + dir * dis;
    float md = ray_box_distance(sp, dir);
    estimated_hit_ts(s, alpha, sp, dir, md, nl, ts);
    if (ts[0] > 0) { ts[0] += dis; ts[2] += dis; }
    if (ts[1] > 0) ts[1] += dis;
}

struct TileAcc {
    float minx = FLT_MAX, miny = FLT_MAX, maxx = -FLT_MAX, maxy = -FLT_MAX;
    f3 avg = {0, 0, 0};
};

static void prepare_ray(const orc_scene* s, float ox, float oy, f3 dir, f3 ro, f3 uo, f3 ori, float alpha,
                        const float nl[3], bool p25, int gid, float* tg, TileAcc& acc, float& hd, float& vd,
                        float ray[4]) {
    f3 sd = normalize((dir + ro * ox) + uo * oy);
    float ts[4];
    sample_t(s, ori, sd, alpha, nl, ts);
    ray[0] = sd.x; ray[1] = sd.y; ray[2] = sd.z; ray[3] = p25 ? ts[1] : ts[0];
    const float rn = 1.0f / 3.0f;
    float min_t = ts[2] * rn, max_t = fmax_(ts[0], ts[1]) * rn;
    tg[gid] = (min_t + max_t) * 0.5f;
    tg[gid + 1] = max_t - min_t;
    tg[gid / 2 + 128] = ts[3];
    if (ray[3] != 0) {
        acc.minx = fmin_(acc.minx, ox); acc.miny = fmin_(acc.miny, oy);
        acc.maxx = fmax_(acc.maxx, ox); acc.maxy = fmax_(acc.maxy, oy);
        acc.avg = acc.avg + ((ts[1] > 0) ? sd * 2.0f : sd);
        float sum_t = ts[0] + ts[1];
        hd += sum_t;
        vd += sum_t;
    }
}

void orc_gather_tiles(const orc_scene* s, const orc_view* v, int px, int py, float* out) {
    const int W = v->width, H = v->height;
    const float neg_logs[3] = {-std::log(0.76f), -std::log(0.75f), -std::log(0.25f)};
    const float* dirs_tab = T("STENCIL_DIRS");
#pragma omp parallel for schedule(dynamic, 4)
    for (int idx = 0; idx < W * H; ++idx) {
        int i = idx / W, j = idx % W;
        float* ob = out + (size_t)idx * 773;
        for (int k = 0; k < 773; ++k) ob[k] = 0;
        float u = 1.0f - ((float)j + (float)px / 8.0f + 0.5f) / (float)W;
        float w = 1.0f - ((float)i + (float)py / 8.0f + 0.5f) / (float)H;
        f3 ori = load3(v->ori), L = load3(v->light_dir);
        f3 fwd = normalize(neg(ori));
        f3 dir = (fwd + (load3(v->right) * (u * 2 - 1))) + (load3(v->up) * (w * 2 - 1));
        f3 ro = f3{-v->right[0] / ((float)W * 4.0f), -v->right[1] / ((float)W * 4.0f), -v->right[2] / ((float)W * 4.0f)};
        f3 uo = f3{-v->up[0] / ((float)H * 4.0f), -v->up[1] / ((float)H * 4.0f), -v->up[2] / ((float)H * 4.0f)};
        float samples[16][4];
        TileAcc acc;
        float hor = 0, vert = 0;
        float* tg = ob + 192 * 3 + 5;
        if (idx == 0) ob[0] *= 1.00001f;
        for (int y = -3, sid = 0, gid = 0, cb = 0; y <= 3; y += 2, cb = (cb + 1) & 1, gid += 16)
            for (int x = -3; x <= 3; x += 2, sid++, gid += 4) {
                bool p25 = ((sid + cb) & 1) != 0;
                float h_ = 0, v_ = 0;
                float r[4], c[4];
                prepare_ray(s, x - 0.5f, y - 0.5f, dir, ro, uo, ori, v->alpha, neg_logs, p25, gid, tg, acc, h_, v_, r);
                const int offs[3][3] = {{1, -1, 2}, {-1, 1, 16}, {1, 1, 18}};
                for (int q = 0; q < 3; ++q) {
                    prepare_ray(s, x + 0.5f * offs[q][0], y + 0.5f * offs[q][1], dir, ro, uo, ori, v->alpha, neg_logs,
                                p25, gid + offs[q][2], tg, acc, h_, v_, c);
                    if ((c[3] != 0 && ((c[3] < r[3]) != p25)) || r[3] == 0)
                        for (int k = 0; k < 4; ++k) r[k] = c[k];
                }
                hor += (x > 0) ? h_ : -h_;
                vert += (y > 0) ? v_ : -v_;
                int fill = sid / 2 + (p25 ? 8 : 0);
                for (int k = 0; k < 4; ++k) samples[fill][k] = r[k];
            }
        if (idx == 0) ob[0] *= 1.00001f;
        if (acc.minx == FLT_MAX) { ob[0] = -1000; continue; }
        Stream st(0, (uint32_t)idx, 0, (uint32_t)v->frame, v->seed);
        f3 bm[3], bl[3];
        basis(acc.avg, 0.0f, st, bm);
        basis(L, 0.0f, st, bl);
        float minx = acc.minx - 0.5f, miny = acc.miny - 0.5f, maxx = acc.maxx + 0.5f, maxy = acc.maxy + 0.5f;
        f3 blc = normalize((dir + ro * minx) + uo * miny), rc = normalize(dir + ro * maxx), uc = normalize(dir + uo * maxy);
        auto sc = [](float x) { return fmax_(-1.0f, fmin_(1.0f, x)); };
        float* go = ob + 192 * 3;
        go[0] = std::acos(sc(dot(bm[0], L)));
        float gbl = std::acos(sc(dot(blc, L)));
        go[1] = std::acos(sc(dot(rc, L))) - gbl;
        go[2] = std::acos(sc(dot(uc, L))) - gbl;
        go[3] = hor;
        go[4] = vert;
        // SetupInputData2: X_Val at [0, 192), X_Val_Hg at [192, 384), X_Val_Sub at [384, 576)
        float* xv = ob;
        float* xh = ob + 192;
        float* xs = ob + 384;
        f3 X = bm[0], Y = bm[1], Z = bm[2];
        for (int k = 0; k < 16; ++k) {
            const float* sm = samples[k];
            if (sm[3] != 0) {
                f3 sd = {sm[0], sm[1], sm[2]};
                f3 sp = ori + sd * sm[3];
                xv[k] = std::log(1.0f + v->alpha * tex3(mip_ptr(s->mips, 0), 256, sp, false) / 64.0f);
                xh[k] = std::log(hg(dot(sd, L), v->g) + 1.0f);
                xs[k] = shadow_tr(s, sp, L, 0);
            } else {
                xv[k] = xh[k] = xs[k] = 0;
            }
        }
        int sid = 0;
        for (int k = 16; k < 192; ++k) {
            while (samples[sid][3] == 0) sid = (sid + 1) & 0xf;
            const float* sm = samples[sid];
            sid = (sid + 1) & 0xf;
            f3 sp = ori + f3{sm[0], sm[1], sm[2]} * sm[3];
            StencilEntry e = stencil(k);
            e.layer += 0.1f;
            int layer = (int)e.layer;
            f3 cur;
            if (e.type >= 4) {
                f3 p = load3(dirs_tab + 3 * k);
                cur = sp + ((X * p.x + Y * p.y + Z * p.z) * e.offset);
            } else {
                cur = sp + L * e.offset;
            }
            xv[k] = std::log(1.0f + v->alpha * tex3(mip_ptr(s->mips, layer), 256 >> layer, cur, false) / 64.0f);
            f3 ms = normalize(cur - sp);
            float radius = (float)(1 << layer) / 256.0f;
            float angle = std::atan(0.5f * radius / e.offset);
            float c1 = dot(X, ms), c2 = dot(L, ms);
            float uu = c1 * 0.5f + 0.5f, uu2 = c2 * 0.5f + 0.5f;
            float vv = angle / (3.1415926535f * 60.0f / 180.0f);
            xh[k] = std::log(tex_lut(s->hg_lut, uu, vv) * tex_lut(s->hg_lut, uu2, vv) + 1.0f);
            xs[k] = shadow_tr(s, cur, L, std::max(layer - 1, 0));
        }
        if (idx == 0) ob[0] *= 1.00001f;
    }
}

// Roberts2, core/vector.cu:179-183: frac(a * n + 0.5) with a = (1/g, 1/g^2, 0)
void orc_roberts2(int n, float out[3]) {
    const float g = 1.32471795724474602596f;
    const float a[3] = {1.0f / g, 1.0f / (g * g), 0.0f};
    for (int c = 0; c < 3; ++c) out[c] = fracf(a[c] * (float)n + 0.5f);
}
// UniformSampleSphere, core/vector.cu:195-205
void orc_uniform_sample_sphere(float ex, float ey, float out[3]) {
    float phi = 2 * 3.14159265359f * ex;
    float ct = 1 - 2 * ey;
    float st = std::sqrt(1 - ct * ct);
    out[0] = st * std::cos(phi);
    out[1] = st * std::sin(phi);
    out[2] = ct;
}
// Image_host::Sample, core/volume.hpp:24-42: bilinear, x first, clamped texels
void orc_image_sample(const float* rgba, int sx, int sy, float u, float v, float out[3]) {
    float px = u * (float)sx - 0.5f, py = v * (float)sy - 0.5f;
    int x = (int)std::floor(px), y = (int)std::floor(py);
    float wx = px - (float)x, wy = py - (float)y;
    auto S = [&](int a, int b, int c) {
        a = a < 0 ? 0 : (a > sx - 1 ? sx - 1 : a);
        b = b < 0 ? 0 : (b > sy - 1 ? sy - 1 : b);
        return rgba[4 * ((size_t)b * sx + a) + c];
    };
    for (int c = 0; c < 3; ++c)
        out[c] = lerpf(lerpf(S(x, y, c), S(x + 1, y, c), wx), lerpf(S(x, y + 1, c), S(x + 1, y + 1, c), wx), wy);
}
// VolumeRender::Render's light choice with an environment map,
// core/volume.cu:494-509 (the coin replaces rand() / RAND_MAX)
void orc_env_light(const orc_scene* s, float coin, int n, float L[3], float C[3]) {
    const float e = s->env_exp;
    const float rate = e * 4 / (e * 4 + fmax_(C[0], fmax_(C[1], C[2])));
    if (!(coin < rate)) {
        for (int c = 0; c < 3; ++c) C[c] = C[c] / (1 - rate);
        return;
    }
    float r[3], d[3], col[3];
    orc_roberts2(n, r);
    orc_uniform_sample_sphere(r[0], r[1], d);
    float u = atan2f(-d[2], d[0]) * (float)(0.5 / 3.1415926) + 0.5f;
    float v = acosf(fmaxf(fminf(d[1], 1.0f), -1.0f)) * (float)(1.0 / 3.1415926);
    orc_image_sample(s->hdri, s->hdri_w, s->hdri_h, u, v, col);
    for (int c = 0; c < 3; ++c) {
        L[c] = d[c];
        C[c] = col[c] * e * 4 / rate;
    }
}
}  // extern "C"
