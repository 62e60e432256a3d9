// volume_kernels.cu -- volume ingest and per-volume resources on the GPU:
// synthetic fBm generation, the 9-level density pyramid, the majorant, the
// empty-space occupancy bricks, the transmittance (TR) mips, the HG phase LUT
// and the baked NEE transmittance grid.
//
// The reference builds the pyramid on the CPU (VolumeRender::Update,
// core/volume.cu:1474-1515) and the TR mips / LUT / baked TR with legacy
// texture + surface references (core/volume.cu:1322-1400, 1535-1696).  Here
// every resource is a plain z-fastest fp32 array in HBM produced by one
// kernel launch per level, on the volume's stream.
#include "kernels.h"

namespace mrp {

// ---------------------------------------------------------------------------
// fBm value noise (synthetic benchmark volumes; not part of the reference).
// PCG-RXS-M-XS lattice hash (Jarzynski & Olano, JCGT 2020), quintic fade.
// ---------------------------------------------------------------------------
MRP_D uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
MRP_D float lattice(uint32_t seed, int ix, int iy, int iz) {
    uint32_t h = pcg(pcg(pcg(pcg(seed) + (uint32_t)ix) + (uint32_t)iy) + (uint32_t)iz);
    return fm((float)(h >> 8), 5.9604644775390625e-8f);
}
MRP_D float quintic(float f) { return fm(fm(fm(f, f), f), fa(fm(f, fs(fm(f, 6.0f), 15.0f)), 10.0f)); }
MRP_D float value_noise(float px, float py, float pz, uint32_t seed) {
    float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    float wx = quintic(fs(px, fx)), wy = quintic(fs(py, fy)), wz = quintic(fs(pz, fz));
    float c00 = lerp(lattice(seed, ix, iy, iz), lattice(seed, ix, iy, iz + 1), wz);
    float c01 = lerp(lattice(seed, ix, iy + 1, iz), lattice(seed, ix, iy + 1, iz + 1), wz);
    float c10 = lerp(lattice(seed, ix + 1, iy, iz), lattice(seed, ix + 1, iy, iz + 1), wz);
    float c11 = lerp(lattice(seed, ix + 1, iy + 1, iz), lattice(seed, ix + 1, iy + 1, iz + 1), wz);
    return lerp(lerp(c00, c01, wy), lerp(c10, c11, wy), wx);
}
MRP_D float fbm_voxel(int R, int x, int y, int z, uint32_t seed, float base_freq, int octaves, float gain) {
    float Rf = (float)R;
    float u = fd(fa((float)x, 0.5f), Rf), v = fd(fa((float)y, 0.5f), Rf), w = fd(fa((float)z, 0.5f), Rf);
    float sum = 0, norm = 0, amp = 1.0f, freq = base_freq;
    for (int o = 0; o < octaves; ++o) {
        sum = fa(sum, fm(amp, value_noise(fm(u, freq), fm(v, freq), fm(w, freq), seed + (uint32_t)o * 1013u)));
        norm = fa(norm, amp);
        amp = fm(amp, gain);
        freq = fm(freq, 2.0f);
    }
    float n = fd(sum, norm);
    float dx = fs(u, 0.5f), dy = fs(v, 0.5f), dz = fs(w, 0.5f);
    float d = fsq(fa(fa(fm(dx, dx), fm(dy, dy)), fm(dz, dz)));
    float t = fd(fs(d, 0.4f), fs(0.32f, 0.4f));
    t = fminf(fmaxf(t, 0.0f), 1.0f);
    float fall = fm(fm(t, t), fs(3.0f, fm(2.0f, t)));
    return fminf(fmaxf(fm(n, fall), 0.0f), 1.0f);
}
// Stores of a grid texel: fp32, or fp16 storage (round to nearest even).
MRP_D void st_f(float* p, float v) { *p = v; }
MRP_D void st_f(__half* p, float v) { *p = __float2half_rn(v); }
template <class T>
__global__ void k_fbm(T* __restrict__ out, int R, uint32_t seed, float base_freq, int octaves, float gain) {
    size_t n = (size_t)R * R * R;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int z = (int)(i % R), y = (int)((i / R) % R), x = (int)(i / ((size_t)R * R));
        st_f(out + i, fbm_voxel(R, x, y, z, seed, base_freq, octaves, gain));
    }
}
// fp32 <-> fp16 storage of a grid (set_data into an fp16 volume, readback).
__global__ void k_narrow(const float* __restrict__ in, size_t n, __half* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = __float2half_rn(in[i]);
}
__global__ void k_widen(const __half* __restrict__ in, size_t n, float* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = __half2float(in[i]);
}

// ---------------------------------------------------------------------------
// Pyramid level from a source grid: the reference's CPU trilinear Sample()
// (border 0, negative values clamped, core/volume.cu:835-863) at texel
// centres u = (i + 0.5) / res (ParallelFill, core/omp.cpp:11-13).
// ---------------------------------------------------------------------------
template <class T>
MRP_D float cpu_fetch(const T* __restrict__ d, int res, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= res || y >= res || z >= res) return 0.0f;
    return fmaxf(0.0f, ldg_f(d + ((size_t)x * res + y) * res + z));
}
template <class T>
__global__ void k_resample(float* __restrict__ out, int res, const T* __restrict__ src, int src_res) {
    size_t n = (size_t)res * res * res;
    float sr = (float)src_res;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int k = (int)(i % res), j = (int)((i / res) % res), q = (int)(i / ((size_t)res * res));
        float u = (float)(((double)q + 0.5) / res), v = (float)(((double)j + 0.5) / res),
              w = (float)(((double)k + 0.5) / res);
        float px = fs(fm(u, sr), 0.5f), py = fs(fm(v, sr), 0.5f), pz = fs(fm(w, sr), 0.5f);
        int x = (int)floorf(px), y = (int)floorf(py), z = (int)floorf(pz);
        float wx = fs(px, (float)x), wy = fs(py, (float)y), wz = fs(pz, (float)z);
        float a = lerp(lerp(cpu_fetch(src, src_res, x, y, z), cpu_fetch(src, src_res, x, y, z + 1), wz),
                       lerp(cpu_fetch(src, src_res, x, y + 1, z), cpu_fetch(src, src_res, x, y + 1, z + 1), wz), wy);
        float b = lerp(lerp(cpu_fetch(src, src_res, x + 1, y, z), cpu_fetch(src, src_res, x + 1, y, z + 1), wz),
                       lerp(cpu_fetch(src, src_res, x + 1, y + 1, z), cpu_fetch(src, src_res, x + 1, y + 1, z + 1), wz), wy);
        out[i] = lerp(a, b, wx);
    }
}

// ---------------------------------------------------------------------------
// max density (the delta-tracking majorant), floored at the reference's
// default 1e-5 (core/volume.hpp:104).  Densities are compared as int bits,
// which orders non-negative floats; negative (SDF) values never win.
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_max_density(const T* __restrict__ d, size_t n, int* __restrict__ out_bits) {
    float m = 0.00001f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, ldg_f(d + i));
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_int(m));
}

// Mip level L and TR level L - 1 side by side per texel, L = 1..4
// (VolumeDev::mip_tr).
__global__ void k_interleave_mip_tr(const float* __restrict__ mips, const float* __restrict__ trs,
                                    float2* __restrict__ out) {
    const int total = mip_tr_offset(5);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int L = 1;
        while (L < 4 && i >= mip_tr_offset(L + 1)) ++L;
        const int j = i - mip_tr_offset(L);
        out[i] = make_float2(mips[mip_offset(L) + j], trs[tr_offset(L - 1) + j]);
    }
}

// The padded mips and TR levels side by side (VolumeDev::pad_pair).
__global__ void k_pair_padded(const float* __restrict__ a, const float* __restrict__ b, float2* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kPadLevelFloats; i += gridDim.x * blockDim.x)
        out[i] = make_float2(a[i], b[i]);
}

// Padded copies of three levels of edge 8, 4, 2 (blockIdx.y picks one): the
// texel of (x, y, z) in [-1, n + 1]^3 is the level's texel under border
// addressing (0 outside) or clamp addressing (nearest edge texel).
__global__ void k_pad_levels(const float* __restrict__ l8, const float* __restrict__ l4, const float* __restrict__ l2,
                             int clamp, float* __restrict__ out) {
    const int n = 8 >> blockIdx.y, P = n + 3;
    const float* src = blockIdx.y == 0 ? l8 : blockIdx.y == 1 ? l4 : l2;
    float* dst = out + pad_offset(n);
    for (int i = threadIdx.x; i < P * P * P; i += blockDim.x) {
        int x = i / (P * P) - 1, y = (i / P) % P - 1, z = i % P - 1;
        float val;
        if (clamp) {
            x = min(max(x, 0), n - 1); y = min(max(y, 0), n - 1); z = min(max(z, 0), n - 1);
            val = src[(x * n + y) * n + z];
        } else {
            const bool in = (unsigned)x < (unsigned)n && (unsigned)y < (unsigned)n && (unsigned)z < (unsigned)n;
            val = in ? src[(x * n + y) * n + z] : 0.0f;
        }
        dst[i] = val;
    }
}

// One warp per grid row (x, y): the lanes scan z, the warp keeps the bounds
// of the nonzero voxels it saw and adds them with six atomics at the end.
template <class T>
__global__ void k_nonzero_bounds(const T* __restrict__ d, int R, int* __restrict__ out6) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x / 32);
    int lo[3] = {R, R, R}, hi[3] = {-1, -1, -1};
    for (long long row = blockIdx.x * (long long)(blockDim.x / 32) + threadIdx.x / 32; row < (long long)R * R;
         row += warps) {
        const T* p = d + row * R;
        int zlo = R, zhi = -1;
        for (int z = lane; z < R; z += 32)
            if (ldg_f(p + z) != 0.0f) { zlo = min(zlo, z); zhi = max(zhi, z); }
        zlo = __reduce_min_sync(0xffffffffu, zlo);
        zhi = __reduce_max_sync(0xffffffffu, zhi);
        if (zhi >= 0) {
            const int x = (int)(row / R), y = (int)(row % R);
            lo[0] = min(lo[0], x); hi[0] = max(hi[0], x);
            lo[1] = min(lo[1], y); hi[1] = max(hi[1], y);
            lo[2] = min(lo[2], zlo); hi[2] = max(hi[2], zhi);
        }
    }
    if (lane == 0 && hi[0] >= 0) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(out6 + a, lo[a]);
            atomicMax(out6 + 3 + a, hi[a]);
        }
    }
}

// ---------------------------------------------------------------------------
// Occupancy bricks for exact empty-space skipping in the first-hit march.
// Brick b covers voxels [b*B, b*B + B) per axis.  A trilinear fetch whose
// base voxel lies in brick b reads voxels base..base+1, i.e. at most one
// voxel past the brick; the brick is marked occupied when any voxel in
// [b*B - 1, b*B + B + 1] holds a non-zero value, one voxel more on each
// side than the fetch needs, so that a base voxel found from a coordinate
// that may be off by less than one voxel still picks a brick whose apron
// holds the whole footprint.  A zero brick therefore guarantees Density() ==
// 0 exactly for every sample whose base voxel is in it or within one voxel
// of it (border texels are 0 by addressing).
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_occupancy(const T* __restrict__ d, int R, int shift, int nb, uint8_t* __restrict__ occ) {
    int total = nb * nb * nb;
    for (int b = blockIdx.x; b < total; b += gridDim.x) {
        int bz = b % nb, by = (b / nb) % nb, bx = b / (nb * nb);
        int B = 1 << shift;
        int x0 = bx * B - 1, y0 = by * B - 1, z0 = bz * B - 1;
        int span = B + 3;
        int any = 0;
        for (int t = threadIdx.x; t < span * span * span && !any; t += blockDim.x) {
            int z = z0 + t % span, y = y0 + (t / span) % span, x = x0 + t / (span * span);
            if ((unsigned)x < (unsigned)R && (unsigned)y < (unsigned)R && (unsigned)z < (unsigned)R)
                any |= ldg_f(d + ((size_t)x * R + y) * R + z) != 0.0f;
        }
        any = __syncthreads_or(any);
        if (threadIdx.x == 0) occ[b] = any ? 1 : 0;
    }
}

// Coarse bricks of 4^3 occupancy bricks (edge 4B): coarse brick C is empty
// when the 64 bricks 4C..4C+3 per axis are.  Their aprons together cover
// voxels [4CB - 1, 4CB + 4B + 1], the coarse brick's own apron, so a zero
// coarse brick carries the same guarantee as a zero brick, over its span.
__global__ void k_occupancy_coarse(const uint8_t* __restrict__ occ, int nb, int nc, uint8_t* __restrict__ out) {
    const int total = nc * nc * nc;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < total; c += gridDim.x * blockDim.x) {
        const int cz = c % nc, cy = (c / nc) % nc, cx = c / (nc * nc);
        int any = 0;
        for (int k = 0; k < 64 && !any; ++k) {
            const int x = 4 * cx + k / 16, y = 4 * cy + (k / 4) % 4, z = 4 * cz + k % 4;
            if (x < nb && y < nb && z < nb) any = occ[(x * nb + y) * nb + z];
        }
        out[c] = any ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// Fill_TR (core/volume.cu:1535-1560): transmittance of TR level `level`
// (res 128>>level) marched 128 steps toward the light through density level
// level+1 with alpha scaled by 1.73^(level+1) (core/volume.cu:1636-1653).
// ---------------------------------------------------------------------------
// src_occ (may be null): 8^3 brick flags of src; empty bricks add exactly 0.
__global__ void k_tr_level(float* __restrict__ out, int res, const float* __restrict__ src,
                           const uint8_t* __restrict__ src_occ, float alpha, f3 L) {
    size_t n = (size_t)res * res * res;
    float rf = (float)res;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int z = (int)(i % res), y = (int)((i / res) % res), x = (int)(i / ((size_t)res * res));
        f3 uv = div(adds(mk3((float)x, (float)y, (float)z), 0.5f), rf);
        f3 ori = subs(uv, 0.5f);
        float dis = ray_box_distance(ori, L);
        float step = fd(dis, 128.0f);
        f3 lp = ori;
        float acc = 0;
        for (int s = 0; s < 128; ++s) {
            lp = add(lp, mul(L, step));
            acc = fa(acc, src_occ ? tex3_occ(src, res, src_occ, (res + 7) >> 3, lp) : tex3<false>(src, res, lp));
        }
        out[i] = fm(1.0f, fm(expf(fm(fm(-acc, alpha), step)), 1.0f));
    }
}

// ---------------------------------------------------------------------------
// Fill_Hg (core/volume.cu:1322-1400): 512x512 LUT of the HG phase averaged
// over a cone, 1024 scrambled-Halton samples per texel.  The digit
// permutations are the reference's (core/volume.cu:1195, from the model
// file), the per-texel shift bn comes from the texel's LUT stream instead of
// a curand draw.
// ---------------------------------------------------------------------------
__constant__ uint32_t c_perm[28];
__constant__ uint32_t c_primes[5] = {2, 3, 5, 7, 11};
__constant__ uint32_t c_prime_sums[5] = {0, 2, 5, 10, 17};

MRP_D float scrambled_radical_inverse(int bi, uint32_t a) {
    const uint32_t base = c_primes[bi], off = c_prime_sums[bi];
    const float inv_base = fd(1.0f, (float)base);
    uint32_t rev = 0;
    float inv_base_n = 1.0f;
    while (a) {
        uint32_t next = a / base;
        uint32_t digit = a - next * base;
        rev = rev * base + c_perm[off + digit];
        inv_base_n = fm(inv_base_n, inv_base);
        a = next;
    }
    return fminf(fm(inv_base_n, fa((float)rev, fd(fm(inv_base, (float)c_perm[off]), fs(1.0f, inv_base)))), 0.99999994f);
}
MRP_D float fracf_(float f) { return fs(f, (float)(long)f); }

__global__ void k_hg_lut(float* __restrict__ lut, float g, uint32_t seed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= kLut || j >= kLut) return;
    float costheta = (float)((((double)(float)i + 0.5) / kLut) * 2.0 - 1.0);
    float aa = (float)(((double)(float)j + 0.5) / kLut);
    float angle = (float)((double)aa * 3.1415926535 * 60.0 / 180.0);
    Stream st(kLutStream, (uint32_t)(j * kLut + i), 0, 0, seed);
    float bn = st.next();
    float h = 0.0f;
    float radius = tanf(angle);
    f3 view = mk3(1.0f, 0.0f, 0.0f);
    f3 dir = mk3(costheta, fsq(fs(1.0f, fm(costheta, costheta))), 0.0f);
    float mis = 0;
    {
        float p = fa(fs(fm(radius, radius), 1.0f), fm(dir.x, dir.x));
        if (p > 0) {
            float sdotl = g > 0 ? dir.x : -dir.x;
            float w = fsq(p);
            float d0 = fd(fmaxf(0.0f, fs(sdotl, w)), radius);
            float d1 = fd(fa(sdotl, w), radius);
            float d = fs(fm(fm(d1, d1), d1), fm(fm(d0, d0), d0));
            mis = fm((float)(d1 > d0), d);
        }
        mis = fminf(fmaxf(mis, 1e-8f), 1.0f);
        float a = fabsf(g);
        double ad = a;
        a = (float)(ad < 0.6 ? 0.0 : (ad < 0.7 ? (ad - 0.6) * 9 : (pow((ad - 0.7) / 0.3, 0.05) * 0.1 + 0.9)));
        mis = fs(1.0f, fd(1.0f, fa(1.0f, fd(fm(a, mis), fs(1.0f, a)))));
    }
    for (uint32_t k = 0; k < 1024; ++k) {
        if (fracf_(fa(scrambled_radical_inverse(4, k), bn)) < mis) {
            float rx = fracf_(fa(scrambled_radical_inverse(0, k), bn));
            float ry = fracf_(fa(scrambled_radical_inverse(1, k), bn));
            f3 l = sample_hg(rx, ry, view, g);
            float sdotl = dot(dir, l);
            float p = fa(fs(fm(radius, radius), 1.0f), fm(sdotl, sdotl));
            if (p <= 0) continue;
            float w = fsq(p);
            float d0 = fs(sdotl, w);
            float d1 = fd(fa(sdotl, w), radius);
            d0 = fd(fmaxf(0.0f, d0), radius);
            float d = fs(fm(fm(d1, d1), d1), fm(fm(d0, d0), d0));
            h = fa(h, fmaxf(0.0f, fd(d, 4.0f)));
        } else {
            float rx = fracf_(fa(scrambled_radical_inverse(0, k), bn));
            float ry = fracf_(fa(scrambled_radical_inverse(1, k), bn));
            float rz = fracf_(fa(scrambled_radical_inverse(2, k), bn));
            float theta = (float)((double)rx * 2.0 * 3.1415926535);
            float phi = (float)acos(2.0 * (double)ry - 1.0);
            float r = powf(rz, fd(1.0f, 3.0f));
            float st_ = sinf(theta), ct = cosf(theta), sp = sinf(phi), cp = cosf(phi);
            float x = fm(fm(fm(radius, r), sp), ct), y = fm(fm(fm(radius, r), sp), st_), z = fm(fm(radius, r), cp);
            f3 rp = add(mk3(x, y, z), dir);
            float c = dot(normalize(rp), view);
            h = fa(h, hg(c, g));
        }
    }
    lut[j * kLut + i] = fd(h, 1024.0f);
}

MRP_D float density(const VolumeDev& v, f3 p) { return density_tex(v, p); }

// Fill_BakeTR (core/volume.cu:1562-1587) over voxels [first, first+count).
// replicate != 0 restarts the voxel's stream for every estimate, as InitRand
// inside the reference's loop does (the estimates are then identical).
__global__ void k_baked_tr(float* __restrict__ out, VolumeDev v, int bake_res, float alpha, f3 L, uint32_t seed,
                           int replicate, int64_t first, int64_t count) {
    float rf = (float)bake_res;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count; q += (int64_t)gridDim.x * blockDim.x) {
        int64_t vi = first + q;
        int x = (int)(vi / ((int64_t)bake_res * bake_res)), y = (int)((vi / bake_res) % bake_res), z = (int)(vi % bake_res);
        f3 uv = div(adds(mk3((float)x, (float)y, (float)z), 0.5f), rf);
        f3 p = subs(uv, 0.5f);
        int cnt = density(v, p) > 0 ? 5 : 2;
        float acc = 0.0f;
        uint32_t hi = (uint32_t)(vi >> 32) * 8u;
        for (int i = 0; i < cnt; ++i) {
            Stream st(kBakeStream, (uint32_t)vi, replicate ? hi : hi + (uint32_t)i, 0, seed);
            float md = ray_box_distance(p, L);
            acc = fa(acc, transmittance(v, st, p, L, md, alpha));
        }
        out[vi] = fm(1.0f, fd(acc, (float)cnt));
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int grid_for(size_t n, int block, int sms) {
    size_t g = (n + block - 1) / block;
    size_t cap = (size_t)sms * 32;
    return (int)(g < cap ? (g ? g : 1) : cap);
}

template <class T>
static cudaError_t fbm_t(T* out, int R, uint32_t seed, float base_freq, int octaves, float gain, int sms,
                         cudaStream_t s) {
    k_fbm<T><<<grid_for((size_t)R * R * R, 256, sms), 256, 0, s>>>(out, R, seed, base_freq, octaves, gain);
    return cudaGetLastError();
}
cudaError_t launch_fbm(float* out, int R, uint32_t seed, float base_freq, int octaves, float gain, int sms,
                       cudaStream_t s) {
    return fbm_t(out, R, seed, base_freq, octaves, gain, sms, s);
}
cudaError_t launch_fbm(__half* out, int R, uint32_t seed, float base_freq, int octaves, float gain, int sms,
                       cudaStream_t s) {
    return fbm_t(out, R, seed, base_freq, octaves, gain, sms, s);
}
cudaError_t launch_narrow(const float* in, size_t n, __half* out, int sms, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_narrow<<<grid_for(n, 256, sms), 256, 0, s>>>(in, n, out);
    return cudaGetLastError();
}
cudaError_t launch_widen(const __half* in, size_t n, float* out, int sms, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_widen<<<grid_for(n, 256, sms), 256, 0, s>>>(in, n, out);
    return cudaGetLastError();
}
cudaError_t launch_resample(float* out, int res, const float* src, int src_res, int sms, cudaStream_t s) {
    k_resample<float><<<grid_for((size_t)res * res * res, 256, sms), 256, 0, s>>>(out, res, src, src_res);
    return cudaGetLastError();
}
cudaError_t launch_resample(float* out, int res, const __half* src, int src_res, int sms, cudaStream_t s) {
    k_resample<__half><<<grid_for((size_t)res * res * res, 256, sms), 256, 0, s>>>(out, res, src, src_res);
    return cudaGetLastError();
}
cudaError_t launch_max_density(const float* d, size_t n, int* out_bits, int sms, cudaStream_t s) {
    k_max_density<float><<<grid_for(n, 256, sms), 256, 0, s>>>(d, n, out_bits);
    return cudaGetLastError();
}
cudaError_t launch_max_density(const __half* d, size_t n, int* out_bits, int sms, cudaStream_t s) {
    k_max_density<__half><<<grid_for(n, 256, sms), 256, 0, s>>>(d, n, out_bits);
    return cudaGetLastError();
}
cudaError_t launch_interleave_mip_tr(const float* mips, const float* trs, float2* out, int sms, cudaStream_t s) {
    k_interleave_mip_tr<<<sms * 8, 256, 0, s>>>(mips, trs, out);
    return cudaGetLastError();
}
cudaError_t launch_pair_padded(const float* mips_pad, const float* trs_pad, float2* out, cudaStream_t s) {
    k_pair_padded<<<(kPadLevelFloats + 255) / 256, 256, 0, s>>>(mips_pad, trs_pad, out);
    return cudaGetLastError();
}
cudaError_t launch_pad_levels(const float* l8, const float* l4, const float* l2, bool clamp, float* out,
                              cudaStream_t s) {
    k_pad_levels<<<dim3(1, 3), 256, 0, s>>>(l8, l4, l2, clamp ? 1 : 0, out);
    return cudaGetLastError();
}
template <class T>
static cudaError_t nonzero_bounds_t(const T* d, int R, int* out6, int sms, cudaStream_t s) {
    long long rows = (long long)R * R;
    int blocks = (int)((rows + 7) / 8 < sms * 16 ? (rows + 7) / 8 : sms * 16);
    k_nonzero_bounds<T><<<blocks, 256, 0, s>>>(d, R, out6);
    return cudaGetLastError();
}
cudaError_t launch_nonzero_bounds(const float* d, int R, int* out6, int sms, cudaStream_t s) {
    return nonzero_bounds_t(d, R, out6, sms, s);
}
cudaError_t launch_nonzero_bounds(const __half* d, int R, int* out6, int sms, cudaStream_t s) {
    return nonzero_bounds_t(d, R, out6, sms, s);
}
template <class T>
static cudaError_t occupancy_t(const T* d, int R, int shift, int nb, uint8_t* occ, int sms, cudaStream_t s) {
    int total = nb * nb * nb;
    k_occupancy<T><<<total < sms * 16 ? total : sms * 16, 256, 0, s>>>(d, R, shift, nb, occ);
    return cudaGetLastError();
}
cudaError_t launch_occupancy(const float* d, int R, int shift, int nb, uint8_t* occ, int sms, cudaStream_t s) {
    return occupancy_t(d, R, shift, nb, occ, sms, s);
}
cudaError_t launch_occupancy(const __half* d, int R, int shift, int nb, uint8_t* occ, int sms, cudaStream_t s) {
    return occupancy_t(d, R, shift, nb, occ, sms, s);
}
cudaError_t launch_occupancy_coarse(const uint8_t* occ, int nb, uint8_t* coarse, int sms, cudaStream_t s) {
    const int nc = (nb + 3) / 4, total = nc * nc * nc;
    k_occupancy_coarse<<<grid_for((size_t)total, 128, sms), 128, 0, s>>>(occ, nb, nc, coarse);
    return cudaGetLastError();
}
cudaError_t launch_tr_level(float* out, int res, const float* src, const uint8_t* src_occ, float alpha,
                            const float L[3], int sms, cudaStream_t s) {
    k_tr_level<<<grid_for((size_t)res * res * res, 128, sms), 128, 0, s>>>(out, res, src, src_occ, alpha,
                                                                           mk3(L[0], L[1], L[2]));
    return cudaGetLastError();
}
cudaError_t set_halton_permutations(const uint32_t perm[28]) {
    return cudaMemcpyToSymbol(c_perm, perm, sizeof(uint32_t) * 28);
}
cudaError_t launch_hg_lut(float* lut, float g, uint32_t seed, cudaStream_t s) {
    k_hg_lut<<<dim3(kLut / 16, kLut / 16), dim3(16, 16), 0, s>>>(lut, g, seed);
    return cudaGetLastError();
}
cudaError_t launch_baked_tr(float* out, const VolumeDev& v, int bake_res, float alpha, const float L[3], uint32_t seed,
                            int replicate, int sms, cudaStream_t s) {
    int64_t total = (int64_t)bake_res * bake_res * bake_res;
    // bounded chunks keep every launch short
    const int64_t chunk = (int64_t)1 << 26;
    for (int64_t first = 0; first < total; first += chunk) {
        int64_t cnt = total - first < chunk ? total - first : chunk;
        k_baked_tr<<<grid_for((size_t)cnt, 128, sms), 128, 0, s>>>(out, v, bake_res, alpha, mk3(L[0], L[1], L[2]),
                                                                   seed, replicate, first, cnt);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace mrp
