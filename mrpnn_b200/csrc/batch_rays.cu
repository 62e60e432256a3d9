// batch_rays.cu -- the reference's batch ray APIs (core/volume.cu:405-479,
// 710-834): GetRadiances (PT or MRPNN for explicit rays), GetSamples (the
// training-data generator) and GetTrs (shadow transmittance x phase).  The
// reference copies its inputs into fresh cudaMallocs each call and polls a
// mapped progress counter; here inputs and outputs may be host or device
// buffers, work runs on the volume's stream, and the kernels are the
// renderer's own (explicit-ray mode of k_trace / k_hit, k_get_samples,
// k_get_trs).
#include <cmath>
#include <vector>

#include "abi_internal.h"

using namespace mrpi;

namespace {
__global__ void k_rgba_to_rgb(const float4* __restrict__ in, int n, float* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = in[i];
    out[3 * i] = a.x;
    out[3 * i + 1] = a.y;
    out[3 * i + 2] = a.z;
}

// Device copies of host inputs for one call, freed at scope exit.
struct Staging {
    std::vector<void*> bufs;
    ~Staging() {
        for (void* p : bufs) mrp::dev_free(p);
    }
    // returns a device pointer to `bytes` of src (host or device)
    cudaError_t in(const void* src, size_t bytes, int is_device, cudaStream_t s, const float** out) {
        if (is_device) { *out = (const float*)src; return cudaSuccess; }
        void* p = nullptr;
        cudaError_t e = mrp::dev_malloc(&p, bytes);
        if (e != cudaSuccess) return e;
        bufs.push_back(p);
        *out = (const float*)p;
        return cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, s);
    }
    cudaError_t scratch(size_t bytes, void** out) {
        cudaError_t e = mrp::dev_malloc(out, bytes);
        if (e == cudaSuccess) bufs.push_back(*out);
        return e;
    }
};
}  // namespace

extern "C" {

mrp_status mrp_get_radiances(mrp_volume* v, const float* ori, const float* dir, int n, const float light_dir[3],
                             const float light_color[3], float alpha, int multi_scatter, float g, int sample_num,
                             mrp_render_type type, float* out3, int is_device) {
    TRY(need_init());
    if (!v || !ori || !dir || !light_dir || !light_color || !out3 || n < 0 || sample_num < 1)
        return fail(MRP_ERR_INVALID, "bad argument");
    if (type == MRP_RPNN) return fail(MRP_ERR_UNSUPPORTED, "RPNN is compiled only with -DCRPNN in the reference");
    if (type != MRP_PT && type != MRP_MRPNN) return fail(MRP_ERR_INVALID, "unknown render type %d", (int)type);
    if (!v->has_data) return fail(MRP_ERR_NOT_READY, "no volume data");
    if (type == MRP_MRPNN && !v->has_pyramid) return fail(MRP_ERR_NOT_READY, "MRPNN needs the pyramid");
    if (n == 0) return MRP_OK;
    if (n > (1 << 26)) return fail(MRP_ERR_INVALID, "%d rays", n);
    mrp_view w{};
    w.width = n;
    w.height = 1;
    for (int c = 0; c < 3; ++c) { w.light_dir[c] = light_dir[c]; w.light_color[c] = light_color[c]; }
    w.alpha = alpha;
    w.g = g;
    w.multi_scatter = multi_scatter;
    w.spp = sample_num;
    Staging S;
    const float *d_ori, *d_dir;
    CU(S.in(ori, (size_t)n * 12, is_device, v->stream, &d_ori));
    CU(S.in(dir, (size_t)n * 12, is_device, v->stream, &d_dir));
    float4* acc;
    CU(S.scratch((size_t)n * sizeof(float4), (void**)&acc));
    VolumeDev d;
    if (type == MRP_PT) {
        if (v->params.nee_mode == 0) {
            // GetRadiances renders through the bake of the current light (MipTr(0, .))
            TRY(update_baked_async(v, light_dir, alpha));
        }
        d = v->dev();
        ViewDev vd = make_view(v, &w, 0, 0);
        vd.ray_ori = d_ori;
        vd.ray_dir = d_dir;
        double* sum3;
        int* first_pos;
        unsigned long long* counter;
        CU(S.scratch((size_t)n * 3 * sizeof(double), (void**)&sum3));
        CU(S.scratch((size_t)n * sizeof(int), (void**)&first_pos));
        CU(S.scratch(sizeof(unsigned long long), (void**)&counter));
        CU(cudaMemsetAsync(sum3, 0, (size_t)n * 3 * sizeof(double), v->stream));
        CU(launch_fill_int(first_pos, n, sample_num, v->stream));
        CU(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), v->stream));
        CU(launch_trace(d, vd, sum3, nullptr, first_pos, counter, mrpi::g.sms, v->stream));
        CU(launch_trace_resolve(sum3, first_pos, n, sample_num, 0, acc, v->stream));
    } else {
        TRY(update_lut_async(v, g));
        TRY(update_tr_async(v, light_dir, alpha));
        d = v->dev();
        ViewDev vd = make_view(v, &w, 0, 0);
        vd.ray_ori = d_ori;
        vd.ray_dir = d_dir;
        int *rc, *rp;
        float *rf, *feat;
        CU(S.scratch(2 * sizeof(int), (void**)&rc));   // records, the march's pixel chunks
        CU(S.scratch((size_t)n * sizeof(int), (void**)&rp));
        CU(S.scratch((size_t)n * 16 * sizeof(float), (void**)&rf));
        CU(S.scratch(tiled_feature_floats(n) * sizeof(float), (void**)&feat));
        HitRecords rec{rc, rp, rf, (size_t)n};
        CU(launch_hit(d, vd, rec, acc, v->stream));
        CU(launch_gather_rec(d, vd, rec, feat, v->params.precision != MRP_FP32, v->stream));
        if (v->params.precision == MRP_FP32) {
            CU(launch_mlp_rec_fp32(d, vd, rec, feat, mrpi::g.d_weights, acc, v->stream));
        } else {
            CU(tc_ensure_scratch(v->tc));
            CU(cudaMemsetAsync(v->tc.d + 1, 0, sizeof(int), v->stream));
            CU(tc_launch_mlp_rec(mrpi::g.tc, v->params.precision == MRP_FP8, d, vd, rec, feat, acc, v->tc, mrpi::g.sms,
                                 v->stream));
        }
    }
    // float4 (L, w) -> float3 L
    float* out;
    CU(S.scratch((size_t)n * 12, (void**)&out));
    k_rgba_to_rgb<<<(n + 255) / 256, 256, 0, v->stream>>>(acc, n, out);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(out3, out, (size_t)n * 12, is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       v->stream));
    CU(cudaStreamSynchronize(v->stream));
    if (type == MRP_MRPNN && v->params.precision != MRP_FP32) {
        int herr = 0;
        CU(cudaMemcpy(&herr, v->tc.d + 1, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) return fail(MRP_ERR_TIMEOUT, "tensor-core MLP: MMA completion wait timed out");
    }
    return MRP_OK;
}

mrp_status mrp_get_samples(mrp_volume* v, const float* alpha, const float* ori, const float* dir,
                           const float* light_dirs, const float* g, const float* scatter, int n,
                           const float light_color[3], int multi_scatter, int sample_num, uint32_t seed, float* out3,
                           int is_device) {
    TRY(need_init());
    if (!v || !alpha || !ori || !dir || !light_dirs || !g || !scatter || !light_color || !out3 || n < 0 ||
        sample_num < 1 || multi_scatter < 1)
        return fail(MRP_ERR_INVALID, "bad argument");
    if (!v->has_data) return fail(MRP_ERR_NOT_READY, "no volume data");
    if (n == 0) return MRP_OK;
    Staging S;
    const float *a, *o, *d, *L, *gg, *sc;
    CU(S.in(alpha, (size_t)n * 4, is_device, v->stream, &a));
    CU(S.in(ori, (size_t)n * 12, is_device, v->stream, &o));
    CU(S.in(dir, (size_t)n * 12, is_device, v->stream, &d));
    CU(S.in(light_dirs, (size_t)n * 12, is_device, v->stream, &L));
    CU(S.in(g, (size_t)n * 4, is_device, v->stream, &gg));
    CU(S.in(scatter, (size_t)n * 4, is_device, v->stream, &sc));
    float* out = out3;
    if (!is_device) CU(S.scratch((size_t)n * 12, (void**)&out));
    CU(launch_get_samples(v->dev(), a, o, d, L, gg, sc, n, light_color, multi_scatter, sample_num, seed, out,
                          v->stream));
    if (!is_device) CU(cudaMemcpyAsync(out3, out, (size_t)n * 12, cudaMemcpyDeviceToHost, v->stream));
    CU(cudaStreamSynchronize(v->stream));
    return MRP_OK;
}

mrp_status mrp_get_trs(mrp_volume* v, float alpha, const float* ori, const float* dir, int n,
                       const float light_dir[3], const float light_color[3], float g, int sample_num, uint32_t seed,
                       float* out3, int is_device) {
    TRY(need_init());
    if (!v || !ori || !dir || !light_dir || !light_color || !out3 || n < 0 || sample_num < 1)
        return fail(MRP_ERR_INVALID, "bad argument");
    if (!v->has_data) return fail(MRP_ERR_NOT_READY, "no volume data");
    if (n == 0) return MRP_OK;
    Staging S;
    const float *o, *d;
    CU(S.in(ori, (size_t)n * 12, is_device, v->stream, &o));
    CU(S.in(dir, (size_t)n * 12, is_device, v->stream, &d));
    float* out = out3;
    if (!is_device) CU(S.scratch((size_t)n * 12, (void**)&out));
    CU(launch_get_trs(v->dev(), alpha, o, d, n, light_dir, light_color, g, sample_num, seed, out, v->stream));
    if (!is_device) CU(cudaMemcpyAsync(out3, out, (size_t)n * 12, cudaMemcpyDeviceToHost, v->stream));
    CU(cudaStreamSynchronize(v->stream));
    return MRP_OK;
}

mrp_status mrp_gather_tiles(mrp_volume* v, const mrp_view* view, int px, int py, float* out, int is_device) {
    TRY(need_init());
    if (!v || !view || !out) return fail(MRP_ERR_INVALID, "null argument");
    if (view->width <= 0 || view->height <= 0 || (long long)view->width * view->height > (1ll << 22))
        return fail(MRP_ERR_INVALID, "tile grid %dx%d", view->width, view->height);
    if (!v->has_pyramid) return fail(MRP_ERR_NOT_READY, "the tile gather needs the pyramid");
    // GatherData updates the LUT and the TR mips first (core/volume.cu:655-657)
    TRY(update_lut_async(v, view->g));
    TRY(update_tr_async(v, view->light_dir, view->alpha));
    const size_t n = (size_t)view->width * view->height, bytes = n * 773 * sizeof(float);
    Staging S;
    float* d_out = out;
    if (!is_device) CU(S.scratch(bytes, (void**)&d_out));
    CU(cudaMemsetAsync(d_out, 0, bytes, v->stream));
    // DeterminateEstimatedHit's thresholds, -logf(0.76 / 0.75 / 0.25), as the
    // host computes them
    const float nl[3] = {-std::log(0.76f), -std::log(0.75f), -std::log(0.25f)};
    ViewDev vd = make_view(v, view, view->frame_offset, 0);
    CU(launch_gather_tiles(v->dev(), vd, px, py, nl, d_out, v->stream));
    if (!is_device) CU(cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, v->stream));
    CU(cudaStreamSynchronize(v->stream));
    return MRP_OK;
}

}  // extern "C"
