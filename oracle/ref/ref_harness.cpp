// ref_harness.cpp -- C entry points over the reference's own render code,
// compiled on the CPU (oracle/Makefile "ref" target -> oracle/_ref/).
//
// TEST INFRASTRUCTURE ONLY.  It exists to pin the oracle restatement
// (oracle/mrpnn_oracle.cpp) to the reference: the functions called below
// (RadiancePredictInternal, SetupInputData, GetSamplePoint,
// GetMatrixFromNormal, NNPredict<MRPNN>, CalculateRadiance, Tr,
// HenyeyGreenstein, SampleHenyeyGreenstein, RayBoxOffset/Distance,
// GetSamples23_, SphereRandom3) are the reference's, unmodified; only the
// CUDA runtime pieces they touch are replaced by ref/shim/.
#include "render.cuh"


thread_local uint3 threadIdx, blockIdx;
thread_local dim3 blockDim, gridDim;

// RadiancePredictInternal and SetupInputData have external linkage in
// core/radiancePredict.cu but no header declaration.
float3 RadiancePredictInternal(float* X_Val, float* X_Val_Sub, float* X_Val_Hg, float gamma, float g,
                               float3 scatterrate);
void SetupInputData(bool active, const float3& pos, const float3& XMain, const float3& YMain, const float3& ZMain,
                    const float3& LXMain, const float3& LightDir, float g, float alpha, float* out_X_Val,
                    float* out_X_Val_Hg, float* out_X_Val_Sub, float& out_gamma);

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
static thread_local uint32_t t_kind = 0, t_id = 0, t_sub = 0, t_frame = 0, t_seed = 0;
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
static void set_stream(uint32_t kind, uint32_t id, uint32_t sub, uint32_t frame, uint32_t seed) {
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
struct Warp {
    std::barrier<> bar{32};
    float f[2][32];
    unsigned u[2][32];
};
static thread_local Warp* t_warp = nullptr;
static thread_local int t_lane = 0, t_phase = 0, t_shfl_slot = -1;
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
// Run body(i, valid) for i in [0, n) as warps of 32 lanes (padding lanes run
// with valid=false and index 0 so that collectives stay complete).
template <class F>
static void run_warps(int n, F body) {
    for (int base = 0; base < n; base += 32) {
        Warp w;
        std::vector<std::thread> lanes;
        for (int l = 0; l < 32; ++l) {
            lanes.emplace_back([&, l] {
                t_warp = &w; t_lane = l; t_phase = 0; t_shfl_slot = -1;
                int i = base + l;
                body(i < n ? i : base, i < n);
                t_warp = nullptr;
            });
        }
        for (auto& t : lanes) t.join();
    }
}

static inline float3 ld3(const float* p) { return float3{p[0], p[1], p[2]}; }
static inline void st3(float* p, float3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

static void bind3(texture<float, cudaTextureType3D, cudaReadModeElementType>& t, const float* d, int n, bool clamp) {
    t.data = d; t.nx = t.ny = t.nz = n;
    t.addressMode[0] = t.addressMode[1] = t.addressMode[2] = clamp ? cudaAddressModeClamp : cudaAddressModeBorder;
}

extern "C" {

// Binds the scene as VolumeRender::Update / Update_TR / UpdateHGLut /
// Update_CachedTR would (core/volume.cu:1456-1531, 1655-1664, 1413-1418,
// 1687-1693).  If baked_tr is given it takes _TR_Mips0, as in PT mode.
void ref_bind_scene(const float* density, int res, float max_density, const float* mips, const float* tr_mips,
                    const float* lut, const float* baked_tr, int baked_res, const float sr[3], float trs,
                    const float sky[3]) {
    bind3(_DensityVolume, density, res, false);
    Resolution = res;
    maxDensity = max_density;
    scatter_rate = ld3(sr);
    tr_scale = trs;
    enviroment_exp = 1.0f;
    texture<float, cudaTextureType3D, cudaReadModeElementType>* m[9] = {&_Mips0, &_Mips1, &_Mips2, &_Mips3, &_Mips4,
                                                                         &_Mips5, &_Mips6, &_Mips7, &_Mips8};
    size_t off = 0;
    for (int i = 0; i < 9; ++i) {
        int r = 256 >> i;
        bind3(*m[i], mips ? mips + off : nullptr, r, false);
        off += (size_t)r * r * r;
    }
    texture<float, cudaTextureType3D, cudaReadModeElementType>* t[8] = {&_TR_Mips0, &_TR_Mips1, &_TR_Mips2, &_TR_Mips3,
                                                                         &_TR_Mips4, &_TR_Mips5, &_TR_Mips6, &_TR_Mips7};
    off = 0;
    for (int i = 0; i < 8; ++i) {
        int r = 128 >> i;
        bind3(*t[i], tr_mips ? tr_mips + off : nullptr, r, true);
        off += (size_t)r * r * r;
    }
    if (baked_tr) bind3(_TR_Mips0, baked_tr, baked_res, true);
    _HGLut.data = lut; _HGLut.nx = 512; _HGLut.ny = 512;
    _HDRI.constant = float4{sky[0], sky[1], sky[2], 1.0f};
    _HDRI.data = nullptr;
}

float ref_hg(float c, float g) { return HenyeyGreenstein(c, g); }
void ref_sample_hg(float e0, float e1, const float v[3], float g, float out[3]) {
    st3(out, SampleHenyeyGreenstein(e0, e1, ld3(v), g));
}
float ref_ray_box_offset(const float p[3], const float d[3]) { return RayBoxOffset(ld3(p), ld3(d)); }
float ref_ray_box_distance(const float p[3], const float d[3]) { return RayBoxDistance(ld3(p), ld3(d)); }
void ref_stencil(int i, float* offset, float* layer, int* type, int* localindex, float dir_out[3]) {
    Offset_Layer_ e = GetSamples23_(i);
    *offset = e.Offset; *layer = e.Layer; *type = e.type; *localindex = e.localindex;
    float3 d = i < 160 ? SphereRandom3(i, 1.0f, float3{1, 0, 0}, float3{0, 1, 0}, float3{0, 0, 1}, 0.0f) : float3{0, 0, 0};
    st3(dir_out, d);
}
float ref_sample_density(int mip, const float pos[3]) {
    return mip < 0 ? Density(ld3(pos)) : MipDensityDynamic(mip, ld3(pos));
}
float ref_shadow_tr(const float pos[3], const float light[3], int mip) {
    return ShadowTerm_TRTex(ld3(pos), ld3(light), float3{1, 0, 0}, float3{1, 1, 1}, 0.0f, mip).x;
}

// RadiancePredictInternal on n feature sets (channel order Val, Sub, Hg),
// lanes of 32 emulated per warp.
void ref_mlp(const float* feat, const float* gamma, float g, const float sr[3], int n, float* out3) {
    run_warps(n, [&](int i, bool valid) {
        float xv[192], xs[192], xh[192];
        for (int k = 0; k < 192; ++k) {
            xv[k] = valid ? feat[(size_t)i * 576 + k] : 0.0f;
            xs[k] = valid ? feat[(size_t)i * 576 + 192 + k] : 0.0f;
            xh[k] = valid ? feat[(size_t)i * 576 + 384 + k] : 0.0f;
        }
        float3 r = RadiancePredictInternal(xv, xs, xh, valid ? gamma[i] : 0.0f, g, ld3(sr));
        if (valid) st3(out3 + 3 * (size_t)i, r);
    });
}

void ref_setup_input(int active, const float pos[3], const float X[3], const float Y[3], const float Z[3],
                     const float LX[3], const float L[3], float g, float alpha, float* feat576, float* gamma) {
    SetupInputData(active != 0, ld3(pos), ld3(X), ld3(Y), ld3(Z), ld3(LX), ld3(L), g, alpha, feat576,
                   feat576 + 384, feat576 + 192, *gamma);
}

int ref_first_hit(const float ori[3], const float dir[3], float alpha, float hit[3]) {
    set_stream(0, 0, 0, 0, 0);
    curandState st;
    curand_init(0, 0, 0, &st);
    float a = alpha;
    float4 r = GetSamplePoint(&st, ld3(ori), ld3(dir), a);
    hit[0] = r.x; hit[1] = r.y; hit[2] = r.z;
    return r.w > 0 ? 1 : 0;
}

void ref_basis(const float v[3], float spread, uint32_t id, uint32_t sub, uint32_t frame, uint32_t seed,
               uint32_t skip, float out9[9]) {
    set_stream(0, id, sub, frame, seed);
    curandState st;
    curand_init(0, 0, 0, &st);
    for (uint32_t i = 0; i < skip; ++i) curand_uniform(&st);
    float3x3 m = GetMatrixFromNormal(&st, ld3(v), spread);
    st3(out9, m.x); st3(out9 + 3, m.y); st3(out9 + 6, m.z);
}

float ref_tr(const float pos[3], const float dir[3], float dis, float alpha, uint32_t id, uint32_t sub,
             uint32_t frame, uint32_t seed, uint32_t kind) {
    set_stream(kind, id, sub, frame, seed);
    curandState st;
    curand_init(0, 0, 0, &st);
    return Tr(&st, ld3(pos), ld3(dir), dis, alpha);
}

// Ray of RenderCamera (core/volume.cu:208-216) for pixel (row, col); this
// wrapper restates those lines (volume.cu does not build on the CPU).
static float3 camera_ray(int W, int H, const float* ori, const float* up, const float* right, int row, int col,
                         uint32_t frame, uint32_t seed) {
    set_stream(0, (uint32_t)(row * W + col), 0, frame, seed);
    curandState st;
    curand_init(0, 0, 0, &st);
    float u = 1 - (col + curand_uniform(&st)) / W;
    float v = 1 - (row + curand_uniform(&st)) / H;
    float3 forward = normalize(-ld3(ori));
    float3 dir = forward + (ld3(right) * (u * 2 - 1)) + (ld3(up) * (v * 2 - 1));
    return normalize(dir);
}

// RenderCamera<true, MRPNN> for a list of pixels: NNPredict per lane, then
// max(0, .).  View layout as orc_view (ints/floats in declaration order).
void ref_predict_pixels(int W, int H, const float ori[3], const float up[3], const float right[3],
                        const float light_dir[3], const float light_color[3], float alpha, float g, uint32_t seed,
                        int frame, const int* pixels, int n, float* rgba) {
    run_warps(n, [&](int q, bool valid) {
        int pix = pixels[q], row = pix / W, col = pix % W;
        float3 dir = camera_ray(W, H, ori, up, right, row, col, (uint32_t)frame, seed);
        set_stream(0, (uint32_t)pix, 0, (uint32_t)frame, seed);
        float4 r = NNPredict<Type::MRPNN>(ld3(ori), dir, ld3(light_dir), ld3(light_color), alpha, g);
        r = max(float4{0, 0, 0, 0}, r);
        if (valid) { rgba[4 * q] = r.x; rgba[4 * q + 1] = r.y; rgba[4 * q + 2] = r.z; rgba[4 * q + 3] = r.w; }
    });
}

// GatherSamples (core/volume.cu:257-282) for tile idx of a W x H tile grid:
// its ray set-up restated here (volume.cu does not build on the CPU), then
// NNGatherSamples as the reference writes it.  The block index marks tile 0
// as the kernel's block (0, 0) / thread (0, 0) for its debug multiplies.
void ref_gather_tile(int W, int H, const float ori[3], const float up[3], const float right[3],
                     const float light_dir[3], float alpha, float g, uint32_t seed, int frame, int px, int py, int idx,
                     float* out773) {
    int i = idx / W, j = idx % W;
    blockIdx.x = idx == 0 ? 0u : 1u;
    blockIdx.y = blockIdx.z = 0u;
    threadIdx.x = threadIdx.y = threadIdx.z = 0u;
    float u = 1.0f - ((float)j + (float)px / 8.0f + 0.5f) / (float)W;
    float v = 1.0f - ((float)i + (float)py / 8.0f + 0.5f) / (float)H;
    float3 forward = normalize(-ld3(ori));
    float3 dir = forward + (ld3(right) * (u * 2 - 1)) + (ld3(up) * (v * 2 - 1));
    float3 right_offset = -ld3(right) / (W * 4.0f);
    float3 up_offset = -ld3(up) / (H * 4.0f);
    set_stream(0, (uint32_t)idx, 0, (uint32_t)frame, seed);
    NNGatherSamples(out773, ld3(ori), dir, ld3(light_dir), right_offset, up_offset, alpha, g);
}

// CalculateRadiance with sampleNum = 1 for sample k of pixel pix (stream sub k).
void ref_trace_sample(int W, int H, const float ori[3], const float up[3], const float right[3],
                      const float light_dir[3], const float light_color[3], float alpha, float g, int multi_scatter,
                      uint32_t seed, int frame, int pix, int k, float out4[4]) {
    int row = pix / W, col = pix % W;
    float3 dir = camera_ray(W, H, ori, up, right, row, col, (uint32_t)frame, seed);
    set_stream(0, (uint32_t)pix, (uint32_t)k, (uint32_t)frame, seed);
    float4 r = CalculateRadiance(ld3(ori), dir, ld3(light_dir), ld3(light_color), alpha, multi_scatter, g, 1);
    out4[0] = r.x; out4[1] = r.y; out4[2] = r.z; out4[3] = r.w;
}

}  // extern "C"
