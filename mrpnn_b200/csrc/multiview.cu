// multiview.cu -- mrp_render_views: n MRPNN views of one volume with one
// batched network launch.  The reference renders views one Render call at a
// time (its data generator loops over cameras, dataGen.cu:246-328); here the
// per-view first hit and gather run back to back on the volume's stream and
// the network of all n views is one persistent tcgen05 launch over a
// segment table (the same kernel the serving loop batches requests with).
// Each view's image equals mrp_render of that view with sample_num 1.
#include <vector>

#include "abi_internal.h"

using namespace mrpi;


extern "C" {

mrp_status mrp_render_views(mrp_volume* v, const mrp_view* views, int n, float* const* outs, int outs_are_device) {
    TRY(need_init());
    if (!v || !views || !outs || n < 1 || n > kTcMaxSegments)
        return fail(MRP_ERR_INVALID, "render_views: 1..%d views with outputs", kTcMaxSegments);
    if (!v->has_pyramid) return fail(MRP_ERR_NOT_READY, "MRPNN needs the pyramid (mrp_volume_update)");
    const mrp_view& w0 = views[0];
    size_t total = 0, feat_floats = 0;
    std::vector<size_t> pix_off(n), feat_off(n);
    for (int i = 0; i < n; ++i) {
        const mrp_view& w = views[i];
        if (!outs[i]) return fail(MRP_ERR_INVALID, "view %d: null output", i);
        if (w.width <= 0 || w.height <= 0 || (long long)w.width * w.height > (1ll << 26))
            return fail(MRP_ERR_INVALID, "view %d: image size %dx%d", i, w.width, w.height);
        for (int c = 0; c < 3; ++c)
            if (w.light_dir[c] != w0.light_dir[c]) return fail(MRP_ERR_INVALID, "views must share the light");
        if (w.alpha != w0.alpha || w.g != w0.g) return fail(MRP_ERR_INVALID, "views must share alpha and g");
        size_t np = (size_t)w.width * w.height;
        pix_off[i] = total;
        feat_off[i] = feat_floats;
        total += np;
        feat_floats += tiled_feature_floats(np);
    }
    // one TR / LUT state for all views (the volume's caches)
    TRY(update_lut_async(v, w0.g));
    TRY(update_tr_async(v, w0.light_dir, w0.alpha));
    // buffers (kept on the volume between calls)
    MultiViewBuffers& B = v->mv;
    if (B.cap_views < kTcMaxSegments) {
        CU(mrp::dev_malloc(&B.rec_count, 2 * kTcMaxSegments * sizeof(int)));   // per view: records, pixel chunks
        CU(mrp::dev_malloc(&B.d_segs, kTcMaxSegments * sizeof(TcSegment)));
        B.cap_views = kTcMaxSegments;
    }
    if (B.cap_pix < total) {
        mrp::dev_free(B.rec_pix); mrp::dev_free(B.rec_f); mrp::dev_free(B.accum);
        B.rec_pix = nullptr; B.rec_f = nullptr; B.accum = nullptr; B.cap_pix = 0;
        CU(mrp::dev_malloc(&B.rec_pix, total * sizeof(int)));
        CU(mrp::dev_malloc(&B.rec_f, total * 16 * sizeof(float)));
        CU(mrp::dev_malloc(&B.accum, total * sizeof(float4)));
        B.cap_pix = total;
    }
    if (B.cap_feat < feat_floats) {
        mrp::dev_free(B.feat);
        B.feat = nullptr;
        B.cap_feat = 0;
        CU(mrp::dev_malloc(&B.feat, feat_floats * sizeof(float)));
        B.cap_feat = feat_floats;
    }
    CU(tc_ensure_scratch(v->tc));
    VolumeDev d = v->dev();
    const bool tc = v->params.precision != MRP_FP32;
    std::vector<TcSegment> segs(n);
    CU(cudaEventRecord(v->ev0, v->stream));
    for (int i = 0; i < n; ++i) {
        size_t np = (size_t)views[i].width * views[i].height;
        // records of view i: SoA arrays with its own capacity np
        HitRecords rec{B.rec_count + 2 * i, B.rec_pix + pix_off[i], B.rec_f + 16 * pix_off[i], np};
        ViewDev vd = make_view(v, &views[i], views[i].frame_offset, 0);
        float4* acc = B.accum + pix_off[i];
        float* ft = B.feat + feat_off[i];
        CU(launch_hit(d, vd, rec, acc, v->stream));
        CU(launch_gather_rec(d, vd, rec, ft, tc, v->stream));
        if (tc) segs[i] = tc_segment(d, vd, rec, ft, acc);
        else CU(launch_mlp_rec_fp32(d, vd, rec, ft, g.d_weights, acc, v->stream));
    }
    CU(cudaEventRecord(v->ev_stage[0], v->stream));
    if (tc) {
        CU(cudaMemcpyAsync(B.d_segs, segs.data(), n * sizeof(TcSegment), cudaMemcpyHostToDevice, v->stream));
        CU(cudaMemsetAsync(v->tc.d + 1, 0, sizeof(int), v->stream));
        CU(tc_launch_mlp_segments(g.tc, v->params.precision == MRP_FP8, B.d_segs, n, v->tc, g.sms, v->stream));
    }
    CU(cudaEventRecord(v->ev_stage[1], v->stream));
    for (int i = 0; i < n; ++i) {
        size_t np = (size_t)views[i].width * views[i].height;
        CU(cudaMemcpyAsync(outs[i], B.accum + pix_off[i], np * sizeof(float4),
                           outs_are_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, v->stream));
    }
    CU(cudaEventRecord(v->ev1, v->stream));
    CU(cudaStreamSynchronize(v->stream));
    if (tc) {
        int herr = 0;
        CU(cudaMemcpy(&herr, v->tc.d + 1, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) return fail(MRP_ERR_TIMEOUT, "tensor-core MLP: MMA completion wait timed out");
    }
    // stage times of this call: hit + gather of all views, network, copies
    CU(cudaEventElapsedTime(&v->stage_ms[0], v->ev0, v->ev_stage[0]));
    CU(cudaEventElapsedTime(&v->stage_ms[1], v->ev_stage[0], v->ev_stage[1]));
    CU(cudaEventElapsedTime(&v->stage_ms[2], v->ev_stage[1], v->ev1));
    CU(cudaEventElapsedTime(&v->last_ms, v->ev0, v->ev1));
    v->stages_valid = true;
    return MRP_OK;
}

}  // extern "C"

namespace mrpi {
void free_multiview(mrp_volume* v) {
    MultiViewBuffers& B = v->mv;
    mrp::dev_free(B.rec_count); mrp::dev_free(B.rec_pix); mrp::dev_free(B.rec_f); mrp::dev_free(B.feat); mrp::dev_free(B.accum);
    mrp::dev_free(B.d_segs);
    B = MultiViewBuffers{};
}
}  // namespace mrpi
