// ref_harness.cpp -- C entry points over the reference's own render code,
// compiled on the CPU (oracle/Makefile "ref" target -> oracle/_ref/).  The
// CUDA stand-ins it relies on are defined in ref_shim_support.cpp.
//
// TEST INFRASTRUCTURE ONLY.  It exists to pin the oracle restatement
// (oracle/mrpnn_oracle.cpp) to the reference: the functions called below
// (RadiancePredictInternal, SetupInputData, GetSamplePoint,
// GetMatrixFromNormal, NNPredict<MRPNN>, CalculateRadiance, Tr,
// HenyeyGreenstein, SampleHenyeyGreenstein, RayBoxOffset/Distance,
// GetSamples23_, SphereRandom3) are the reference's, unmodified; only the
// CUDA runtime pieces they touch are replaced by ref/shim/.
#include "render.cuh"


// RadiancePredictInternal and SetupInputData have external linkage in
// core/radiancePredict.cu but no header declaration.
float3 RadiancePredictInternal(float* X_Val, float* X_Val_Sub, float* X_Val_Hg, float gamma, float g,
                               float3 scatterrate);
void SetupInputData(bool active, const float3& pos, const float3& XMain, const float3& YMain, const float3& ZMain,
                    const float3& LXMain, const float3& LightDir, float g, float alpha, float* out_X_Val,
                    float* out_X_Val_Hg, float* out_X_Val_Sub, float& out_gamma);

#include "ref_support.h"

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
                    const float sky[3], const float* hdri, int hdri_w, int hdri_h, float env_exp) {
    bind3(_DensityVolume, density, res, false);
    Resolution = res;
    maxDensity = max_density;
    scatter_rate = ld3(sr);
    tr_scale = trs;
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
    // SetHDRI (core/volume.cu:1696-1728) binds the map with wrap addressing
    // and SetEnvExp sets enviroment_exp; without a map the constant sky
    // stands in for the (otherwise unbound, zero) environment
    _HDRI.constant = float4{sky[0], sky[1], sky[2], 1.0f};
    _HDRI.data = reinterpret_cast<const float4*>(hdri);
    _HDRI.nx = hdri ? hdri_w : 0;
    _HDRI.ny = hdri ? hdri_h : 0;
    enviroment_exp = hdri ? env_exp : 1.0f;
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
    ref_set_stream(0, 0, 0, 0, 0);
    curandState st;
    curand_init(0, 0, 0, &st);
    float a = alpha;
    float4 r = GetSamplePoint(&st, ld3(ori), ld3(dir), a);
    hit[0] = r.x; hit[1] = r.y; hit[2] = r.z;
    return r.w > 0 ? 1 : 0;
}

void ref_basis(const float v[3], float spread, uint32_t id, uint32_t sub, uint32_t frame, uint32_t seed,
               uint32_t skip, float out9[9]) {
    ref_set_stream(0, id, sub, frame, seed);
    curandState st;
    curand_init(0, 0, 0, &st);
    for (uint32_t i = 0; i < skip; ++i) curand_uniform(&st);
    float3x3 m = GetMatrixFromNormal(&st, ld3(v), spread);
    st3(out9, m.x); st3(out9 + 3, m.y); st3(out9 + 6, m.z);
}

float ref_tr(const float pos[3], const float dir[3], float dis, float alpha, uint32_t id, uint32_t sub,
             uint32_t frame, uint32_t seed, uint32_t kind) {
    ref_set_stream(kind, id, sub, frame, seed);
    curandState st;
    curand_init(0, 0, 0, &st);
    return Tr(&st, ld3(pos), ld3(dir), dis, alpha);
}

// Ray of RenderCamera (core/volume.cu:208-216) for pixel (row, col); this
// wrapper restates those lines (volume.cu does not build on the CPU).
static float3 camera_ray(int W, int H, const float* ori, const float* up, const float* right, int row, int col,
                         uint32_t frame, uint32_t seed) {
    ref_set_stream(0, (uint32_t)(row * W + col), 0, frame, seed);
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
        ref_set_stream(0, (uint32_t)pix, 0, (uint32_t)frame, seed);
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
    ref_set_stream(0, (uint32_t)idx, 0, (uint32_t)frame, seed);
    NNGatherSamples(out773, ld3(ori), dir, ld3(light_dir), right_offset, up_offset, alpha, g);
}

// CalculateRadiance with sampleNum = 1 for sample k of pixel pix (stream sub k).
void ref_trace_sample(int W, int H, const float ori[3], const float up[3], const float right[3],
                      const float light_dir[3], const float light_color[3], float alpha, float g, int multi_scatter,
                      uint32_t seed, int frame, int pix, int k, float out4[4]) {
    int row = pix / W, col = pix % W;
    float3 dir = camera_ray(W, H, ori, up, right, row, col, (uint32_t)frame, seed);
    ref_set_stream(0, (uint32_t)pix, (uint32_t)k, (uint32_t)frame, seed);
    float4 r = CalculateRadiance(ld3(ori), dir, ld3(light_dir), ld3(light_color), alpha, multi_scatter, g, 1);
    out4[0] = r.x; out4[1] = r.y; out4[2] = r.z; out4[3] = r.w;
}

}  // extern "C"
