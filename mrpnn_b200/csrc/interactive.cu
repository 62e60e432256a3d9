// interactive.cu -- one frame of the reference's real-time viewer path,
// VolumeRender::Render(float3* target, Histogram*, unsigned* target2, ...)
// (core/volume.cu:550-628): the interactive RenderCamera (core/volume.cu:57-
// 196; checkerboard rendering, per-pixel running mean and radiance histogram
// for the tracer), then Denoise (histogram-weighted 11 x 11 filter,
// core/volume.cu:285-330) or ReprojectionDenoise (core/volume.cu:332-353),
// exposure, Gamma / ACES tone mapping (core/render.cuh:1144-1236) and the
// RGBA8 pack.  target, histo and rgba8 are caller-owned buffers, as in the
// reference; frame number, flip and exposure are arguments instead of
// __device__ globals.
#include "abi_internal.h"
#include "tracing.cuh"

using namespace mrpi;

namespace {

constexpr int kHisto = 10;   // HISTO_SIZE (core/volume.hpp:12)

// float3 x float3x3 rows (float3x3::operator*, core/vector.cu:261-263)
MRP_D f3 mat3(f3 r0, f3 r1, f3 r2, f3 v) { return mk3(dot(r0, v), dot(r1, v), dot(r2, v)); }
MRP_D f3 lerp3(f3 a, f3 b, float t) { return mk3(lerp(a.x, b.x, t), lerp(a.y, b.y, t), lerp(a.z, b.z, t)); }
MRP_D f3 pow3(f3 a, float e) { return mk3(powf(a.x, e), powf(a.y, e), powf(a.z, e)); }
MRP_D f3 gamma_tone(f3 c) { return pow3(c, fd(1.0f, 2.2f)); }

// ACES (core/render.cuh:1157-1236), same constants and operation order
MRP_D f3 aces_tone(f3 color) {
    const f3 AP1_XYZ0 = mk3(0.6624541811f, 0.1340042065f, 0.1561876870f);
    const f3 AP1_XYZ1 = mk3(0.2722287168f, 0.6740817658f, 0.0536895174f);
    const f3 AP1_XYZ2 = mk3(-0.0055746495f, 0.0040607335f, 1.0103391003f);
    f3 aces = mat3(mk3(0.4397010f, 0.3829780f, 0.1773350f), mk3(0.0897923f, 0.8134230f, 0.0967616f),
                   mk3(0.0175440f, 0.1115440f, 0.8707040f), color);
    const f3 Y = mk3(0.272229f, 0.674082f, 0.0536895f);
    f3 cg = mat3(mk3(1.4514393161f, -0.2365107469f, -0.2149285693f), mk3(-0.0765537734f, 1.1762296998f, -0.0996759264f),
                 mk3(0.0083161484f, -0.0060324498f, 0.9977163014f), aces);
    float tmp = dot(cg, Y);
    cg = lerp3(mk3(tmp, tmp, tmp), cg, 0.96f);
    const float a = 278.5085f, b = 10.7772f, c = 293.6045f, d = 88.7122f, e = 80.6889f;
    f3 x = cg;
    f3 num = mul(x, adds(mul(x, a), b));
    f3 den = adds(mul(x, adds(mul(x, c), d)), e);
    f3 post = mk3(fd(num.x, den.x), fd(num.y, den.y), fd(num.z, den.z));
    // darkSurround_to_dimSurround
    f3 XYZ = mat3(AP1_XYZ0, AP1_XYZ1, AP1_XYZ2, post);
    float divisor = fmaxf(dot(XYZ, mk3(1, 1, 1)), 1e-4f);
    f3 xyY = mk3(fd(XYZ.x, divisor), fd(XYZ.y, divisor), XYZ.y);
    xyY.z = fminf(fmaxf(xyY.z, 0.0f), 65504.0f);
    xyY.z = powf(xyY.z, 0.9811f);
    float m = fd(xyY.z, fmaxf(xyY.y, 1e-4f));
    XYZ = mk3(fm(xyY.x, m), xyY.z, fm(fs(fs(1.0f, xyY.x), xyY.y), m));
    f3 lin = mat3(mk3(1.6410233797f, -0.3248032942f, -0.2364246952f), mk3(-0.6636628587f, 1.6153315917f, 0.0167563477f),
                  mk3(0.0117218943f, -0.0082844420f, 0.9883948585f), XYZ);
    tmp = dot(lin, Y);
    lin = lerp3(mk3(tmp, tmp, tmp), lin, 0.93f);
    XYZ = mat3(AP1_XYZ0, AP1_XYZ1, AP1_XYZ2, lin);
    XYZ = mat3(mk3(0.98722400f, -0.00611327f, 0.0159533f), mk3(-0.00759836f, 1.00186000f, 0.0053302f),
               mk3(0.00307257f, -0.00509595f, 1.0816800f), XYZ);
    lin = mat3(mk3(3.2409699419f, -1.5373831776f, -0.4986107603f), mk3(-0.9692436363f, 1.8759675015f, 0.0415550574f),
               mk3(0.0556300797f, -0.2039769589f, 1.0569715142f), XYZ);
    return gamma_tone(lin);
}

MRP_D float saturate1(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }
MRP_D uint32_t pack_rgba8(f3 val) {
    uint32_t r = (uint32_t)(255.0f * saturate1(val.x)), g_ = (uint32_t)(255.0f * saturate1(val.y)),
             b = (uint32_t)(255.0f * saturate1(val.z));
    return 0xff000000u | (r << 16) | (g_ << 8) | b;
}
MRP_D f3 tone(f3 val, int type) { return type == 1 ? gamma_tone(val) : type == 2 ? aces_tone(val) : val; }

MRP_D f3 ld_t(const float* t, int i) { return mk3(t[3 * i], t[3 * i + 1], t[3 * i + 2]); }
MRP_D void st_t(float* t, int i, f3 v) { t[3 * i] = v.x; t[3 * i + 1] = v.y; t[3 * i + 2] = v.z; }

// UnRoll (core/volume.cu:230-234): (row, col) clamped to the image
MRP_D int unroll(int row, int col, int W, int H) {
    col = min(max(0, col), W - 1);
    row = min(max(0, row), H - 1);
    return col + W * row;
}

// Compare (core/volume.cu:236-254): chi-square distance of two histograms
MRP_D float compare(const mrp_histogram& x, const mrp_histogram& y) {
    float nx = x.total, ny = y.total;
    float sy = fsq(fd(ny, nx)), sx = fsq(fd(nx, ny));
    float p = 0, res = 0;
    for (int i = 0; i < 3 * kHisto; ++i) {
        float hx = x.bin[i], hy = y.bin[i];
        if (hx != 0 || hy != 0) {
            p = fa(p, 1.0f);
            float t = fs(fm(sy, hx), fm(sx, hy));
            res = fa(res, fd(fm(t, t), fa(hx, hy)));
        }
    }
    return p == 0 ? 0.0f : fd(res, p);
}

// Tracer frame: one sample per selected pixel, running mean and histogram
// (RenderCamera<false>, core/volume.cu:103-129).
__global__ void k_frame_pt(VolumeDev v, ViewDev w, int fnum, float* __restrict__ target,
                           mrp_histogram* __restrict__ histo) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= w.width * w.height) return;
    int row = idx / w.width, col = idx % w.width;
    if (!pixel_selected(w, row, col)) return;
    f3 dir = normalize(camera_ray_dir(w, row, col));   // CalculateRadiance normalizes again (core/render.cuh:540)
    f3 L = normalize(w.light_dir);
    float dis = ray_box_offset(w.ori, dir);
    f3 res = dis < 0 ? sky_radiance(v, dir) : trace_sample(v, w, idx, 0, w.ori, dir, dis, L, nullptr);
    res = mk3(fmaxf(0.0f, res.x), fmaxf(0.0f, res.y), fmaxf(0.0f, res.z));
    mrp_histogram h = histo[idx];
    if (fnum == 0) h = mrp_histogram{};
    float rate = fd(1.0f, (float)(1 + fnum));
    st_t(target, idx, lerp3(ld_t(target, idx), res, rate));
    res = mk3(fd(res.x, fa(res.x, 1.0f)), fd(res.y, fa(res.y, 1.0f)), fd(res.z, fa(res.z, 1.0f)));
    h.total = fa(h.total, 1.0f);
    int bx = (int)floorf(fm(fminf(res.x, 0.999f), (float)kHisto));
    int by = (int)floorf(fm(fminf(res.y, 0.999f), (float)kHisto));
    int bz = (int)floorf(fm(fminf(res.z, 0.999f), (float)kHisto));
    h.bin[bx] = fa(h.bin[bx], 1.0f);
    h.bin[by + kHisto] = fa(h.bin[by + kHisto], 1.0f);
    h.bin[bz + 2 * kHisto] = fa(h.bin[bz + 2 * kHisto], 1.0f);
    float l = dot(res, mk3(1, 1, 1));
    h.x = lerp(h.x, l, rate);
    h.x2 = lerp(h.x2, fm(l, l), rate);
    histo[idx] = h;
}

// Predictor frame: target = max(0, NNPredict) at the selected pixels
// (RenderCamera<true>, core/volume.cu:131-150; the reprojection there ends
// in target = res).
__global__ void k_frame_mrpnn(const float4* __restrict__ accum, ViewDev w, float* __restrict__ target) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= w.width * w.height) return;
    if (!pixel_selected(w, idx / w.width, idx % w.width)) return;
    float4 a = accum[idx];
    st_t(target, idx, mk3(fmaxf(0.0f, a.x), fmaxf(0.0f, a.y), fmaxf(0.0f, a.z)));
}

// Denoise<denoise> (PT) / ReprojectionDenoise (MRPNN), exposure, tone map, RGBA8.
__global__ void k_frame_finish(const float* __restrict__ target, mrp_histogram* __restrict__ histo,
                               uint32_t* __restrict__ rgba8, int W, int H, int frame_num, int flip, int predict,
                               int denoise, float exposure, int tone_type) {
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= W * H) return;
    int row = id / W, col = id % W;
    f3 res;
    if (predict) {
        f3 t = ld_t(target, id);
        histo[id].total = t.x;
        histo[id].x = t.y;
        histo[id].x2 = t.z;
        res = t;
    } else if (frame_num == 0) {
        if ((((row + flip) % 2) + col) % 2 == 0) {
            res = ld_t(target, id);
        } else {
            res = add(add(add(ld_t(target, unroll(row - 1, col, W, H)), ld_t(target, unroll(row + 1, col, W, H))),
                          ld_t(target, unroll(row, col - 1, W, H))),
                      ld_t(target, unroll(row, col + 1, W, H)));
            res = mk3(fd(res.x, 4.0f), fd(res.y, 4.0f), fd(res.z, 4.0f));
        }
    } else {
        const mrp_histogram c = histo[id];
        float variance = fabsf(fs(c.x2, fm(c.x, c.x)));
        if (denoise && variance > 0.01) {
            res = mk3(0, 0, 0);
            float ws = 0;
            for (int i = -5; i <= 5; ++i)
                for (int j = -5; j <= 5; ++j) {
                    int t = unroll(row + i, col + j, W, H);
                    float wgt = (float)fmax(0.0, 1.0 - 1.2 * (double)compare(c, histo[t]));
                    res = add(res, mul(ld_t(target, t), wgt));
                    ws = fa(ws, wgt);
                }
            res = mk3(fd(res.x, ws), fd(res.y, ws), fd(res.z, ws));
        } else {
            res = ld_t(target, id);
        }
    }
    rgba8[id] = pack_rgba8(tone(mul(res, exposure), tone_type));
}

}  // namespace

extern "C" {

mrp_status mrp_render_interactive(mrp_volume* v, const mrp_view* view, mrp_render_type type, int frame_num,
                                  int checkerboard, int flip, int tone_type, int denoise, float exposure,
                                  float* target, mrp_histogram* histo, uint32_t* rgba8, int rgba8_is_device) {
    TRY(need_init());
    if (!v || !view || !target || !histo || !rgba8 || frame_num < 0) return fail(MRP_ERR_INVALID, "bad argument");
    if (type == MRP_RPNN) return fail(MRP_ERR_UNSUPPORTED, "RPNN is compiled only with -DCRPNN in the reference");
    if (type != MRP_PT && type != MRP_MRPNN) return fail(MRP_ERR_INVALID, "unknown render type %d", (int)type);
    if (view->width <= 0 || view->height <= 0 || (long long)view->width * view->height > (1ll << 26))
        return fail(MRP_ERR_INVALID, "image size %dx%d", view->width, view->height);
    if (!v->has_data) return fail(MRP_ERR_NOT_READY, "no volume data");
    if (type == MRP_MRPNN && !v->has_pyramid) return fail(MRP_ERR_NOT_READY, "MRPNN needs the pyramid");
    if (v->async_inflight) TRY(mrp_render_wait(v, 0));   // started renders may still read accum
    const int W = view->width, H = view->height, npix = W * H;
    const int fnum = checkerboard ? frame_num / 2 : frame_num;
    // the viewer's predictor frame with an environment map lights it from the
    // map or the sun (core/volume.cu:552-567); the map's direction index
    // advances every frame (rand_cpu++, core/volume.cu:579)
    mrp_view vw = *view;
    if (type == MRP_MRPNN && v->hdri)
        env_light_for_launch(v, (uint32_t)view->frame_offset, view->seed, vw.light_dir, vw.light_color);
    view = &vw;
    ViewDev vd = make_view(v, view, view->frame_offset, 0);
    vd.cam_mode = 1;
    vd.checker = checkerboard ? 1 : 0;
    vd.flip = flip & 1;
    const bool predict = type == MRP_MRPNN;
    uint32_t* out = rgba8;
    uint32_t* tmp = nullptr;
    if (!rgba8_is_device) {
        CU(mrp::dev_malloc_async(&tmp, (size_t)npix * 4, v->stream));
        out = tmp;
    }
    mrp_status st = MRP_OK;
    auto run = [&]() -> mrp_status {
        if (predict) {
            TRY(update_lut_async(v, view->g));
            TRY(update_tr_async(v, view->light_dir, view->alpha));
            TRY(ensure_predictor_buffers(v, (size_t)npix));
            TRY(ensure_accum(v, (size_t)npix));
            VolumeDev d = v->dev();
            HitRecords rec = v->records();
            CU(launch_hit(d, vd, rec, v->accum, v->stream));
            CU(launch_gather_rec(d, vd, rec, v->feat, v->params.precision != MRP_FP32, v->stream));
            if (v->params.precision == MRP_FP32) {
                CU(launch_mlp_rec_fp32(d, vd, rec, v->feat, g.d_weights, v->accum, v->stream));
            } else {
                CU(cudaMemsetAsync(v->tc.d + 1, 0, sizeof(int), v->stream));
                CU(tc_launch_mlp_rec(g.tc, v->params.precision == MRP_FP8, d, vd, rec, v->feat, v->accum, v->tc,
                                     g.sms, v->stream));
            }
            k_frame_mrpnn<<<(npix + 255) / 256, 256, 0, v->stream>>>(v->accum, vd, target);
            CU(cudaGetLastError());
        } else {
            if (v->params.nee_mode == 0) TRY(update_baked_async(v, view->light_dir, view->alpha));
            k_frame_pt<<<(npix + 127) / 128, 128, 0, v->stream>>>(v->dev(), vd, fnum, target, histo);
            CU(cudaGetLastError());
        }
        k_frame_finish<<<(npix + 255) / 256, 256, 0, v->stream>>>(target, histo, out, W, H, frame_num, flip & 1,
                                                                   predict ? 1 : 0, denoise ? 1 : 0, exposure,
                                                                   tone_type);
        CU(cudaGetLastError());
        if (tmp) CU(cudaMemcpyAsync(rgba8, tmp, (size_t)npix * 4, cudaMemcpyDeviceToHost, v->stream));
        CU(cudaStreamSynchronize(v->stream));
        return MRP_OK;
    };
    st = run();
    ++v->hdri_light_n;
    if (tmp) mrp::dev_free_async(tmp, v->stream);
    if (st != MRP_OK) return st;
    if (predict && v->params.precision != MRP_FP32) {
        int herr = 0;
        CU(cudaMemcpy(&herr, v->tc.d + 1, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) return fail(MRP_ERR_TIMEOUT, "tensor-core MLP: MMA completion wait timed out");
    }
    return MRP_OK;
}

}  // extern "C"
