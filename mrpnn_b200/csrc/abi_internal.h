// abi_internal.h -- state shared by the C ABI's translation units (abi.cu,
// serve.cu): the library singleton, the volume handle, error reporting.
#pragma once
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mrpnn.h"
#include "kernels.h"
#include "mlp_tc.h"

struct mrp_volume;
namespace mrpi {
using namespace mrp;

// Device buffers of mrp_render_views, kept per volume between calls (grown,
// never shrunk): records and tiled features of all views concatenated.
struct MultiViewBuffers {
    int* rec_count = nullptr;   // [kTcMaxSegments]
    int* rec_pix = nullptr;     // [total pixels]
    float* rec_f = nullptr;     // [16 x total pixels]
    float* feat = nullptr;
    float4* accum = nullptr;    // [total pixels]
    TcSegment* d_segs = nullptr;
    size_t cap_pix = 0, cap_feat = 0;
    int cap_views = 0;
};
void free_multiview(mrp_volume* v);

// Sets the calling thread's last error (mrp_last_error) and returns s.
mrp_status fail(mrp_status s, const char* fmt, ...);

struct Lib {
    std::mutex mu;
    bool ready = false;
    int device = -1;
    int sms = 148;
    cudaStream_t stream = nullptr;   // for handle-less calls
    std::map<std::string, std::vector<float>> model;
    float* d_weights = nullptr;      // packed fp32 weights + transposed copies (common.cuh layout, kWeightCountDev)
    std::vector<float> h_weights;
    TcWeights tc;                    // tensor-core weight images
    // scratch for handle-less parity calls
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
};
extern Lib g;

// Device view of one camera launch (RenderCamera's arguments).
ViewDev make_view(const mrp_volume* v, const mrp_view* w, int frame, int mean_k);
// Fill_TR for the 8 TR levels of a pyramid into trs (kTrFloats floats).
cudaError_t build_tr_levels(float* trs, const float* mips, const uint8_t* mip_occ, const float L[3], float alpha,
                            cudaStream_t s);

// Per-volume caches of the predictor, queued on the volume's stream: the HG
// LUT for g (UpdateHGLut) and the TR mips for (light, alpha) (Update_TR).
mrp_status update_lut_async(mrp_volume* v, float g);
mrp_status update_tr_async(mrp_volume* v, const float L[3], float alpha);
// Staged-predictor records / features and the running-mean image of a volume,
// grown to npix pixels.
mrp_status ensure_predictor_buffers(mrp_volume* v, size_t npix);
mrp_status ensure_accum(mrp_volume* v, size_t npix);
// The baked NEE grid for (light, alpha) (Update_CachedTR), on the volume's stream.
mrp_status update_baked_async(mrp_volume* v, const float L[3], float alpha);

inline mrp_status need_init() {
    if (!g.ready) return fail(MRP_ERR_NOT_READY, "mrp_init has not been called");
    return MRP_OK;
}

}  // namespace mrpi

#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return mrpi::fail(e_ == cudaErrorMemoryAllocation ? MRP_ERR_OOM : MRP_ERR_CUDA, "%s: %s (%s:%d)", #call, \
                              cudaGetErrorString(e_), __FILE__, __LINE__);                         \
    } while (0)
#define TRY(call)                                                                                  \
    do {                                                                                           \
        mrp_status s_ = (call);                                                                    \
        if (s_ != MRP_OK) return s_;                                                               \
    } while (0)

// ---------------------------------------------------------------------------
// volume handle
// ---------------------------------------------------------------------------
struct mrp_volume {
    using VolumeDev = mrp::VolumeDev;
    using HitRecords = mrp::HitRecords;
    using TcScratch = mrp::TcScratch;
    int res = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_stage[2] = {nullptr, nullptr};   // stage boundaries of the last launch
    float last_ms = 0.0f;
    float stage_ms[3] = {0, 0, 0};
    bool stages_valid = false;
    float* density = nullptr;       // fp32 storage, or
    __half* density_h = nullptr;    // fp16 storage (MRP_STORAGE_FP16)
    float* mips = nullptr;
    float* trs = nullptr;
    float* lut = nullptr;
    float* baked = nullptr;
    int baked_alloc_res = 0;
    uint8_t* occ = nullptr;
    uint8_t* mip_occ = nullptr;   // bricks of mip levels 0..kOccMips-1
    int occ_shift = 3, occ_res = 0;
    uint8_t* occ2 = nullptr;      // coarse occupancy (4^3 bricks each), built with occ
    int occ2_res = 0;
    int* d_maxbits = nullptr;
    float* mips_pad = nullptr;    // padded mips 5..7 (pad_offset layout), built with the pyramid
    float* trs_pad = nullptr;     // padded TR levels 4..6, built with the TR levels
    float2* mip_tr = nullptr;     // (mip L, TR L - 1) texel pairs, L = 1..4, built with the TR levels
    float2* pad_pair = nullptr;   // (padded mip, padded TR) pairs, built with the TR levels
    int* d_bounds = nullptr;      // nonzero-voxel index bounds (6 ints) of the last update
    int nz_bounds[6] = {0, 0, 0, -1, -1, -1};
    bool has_bounds = false;
    bool has_data = false, has_pyramid = false, has_lut = false, has_tr = false, has_baked = false;
    bool max_override = false;
    float max_density = 0.00001f;
    float lut_g = NAN, tr_alpha = NAN, tr_light[3] = {NAN, NAN, NAN};
    float bk_alpha = NAN, bk_light[3] = {NAN, NAN, NAN};
    int bk_res = 0;
    uint32_t lut_seed = 0, bk_seed = 0;
    mrp_params params;
    // render buffers
    float4* accum = nullptr;
    size_t accum_pix = 0;
    // mrp_render_start: results alternate between accum and accum_alt, and
    // are copied out on stream_copy while the next render computes
    cudaStream_t stream_copy = nullptr;
    float4* accum_alt = nullptr;
    size_t accum_alt_pix = 0;
    cudaEvent_t ev_done[2] = {nullptr, nullptr};     // compute into slot s finished
    cudaEvent_t ev_copied[2] = {nullptr, nullptr};   // copy out of slot s finished
    int async_slot = 0;
    int async_inflight = 0;
    bool async_tc = false;   // a tensor-core network ran since the last wait
    double* sum3 = nullptr;
    int* first_pos = nullptr;
    unsigned long long* counter = nullptr;
    size_t trace_pix = 0;
    // staged predictor buffers (records of hit pixels, tiled features)
    int* rec_count = nullptr;
    int* rec_pix = nullptr;
    float* rec_f = nullptr;
    float* feat = nullptr;
    size_t rec_cap = 0;
    // environment map of SetHDRI (RGBA float rows), device and host copies
    float4* hdri = nullptr;
    int hdri_w = 0, hdri_h = 0;
    std::vector<float> hdri_host;
    int hdri_light_n = 0;   // Roberts2 index of the map's light direction (the reference's rand_cpu)
    // the density grid as a texture for the tracer's hardware filter (built
    // on first use, dropped when the grid changes)
    cudaArray_t dens_arr = nullptr;
    cudaTextureObject_t dens_tex = 0;
    mrp::GtexLevel baked_gtex;   // the baked NEE grid as a texture (tracer_filter), refilled after each bake
    bool baked_gtex_ok = false;
    // the pyramid, TR levels and LUT as textures for the fp16-feature gather
    // (gather_filter): allocated on first use, refreshed in place whenever a
    // builder rewrites the linear copy (gtex_dirty: 1 mips, 2 TR, 4 LUT)
    mrp::GtexLevel gmip0, gtr0, gpair[mrp::kGtexPairs], glut;
    bool gtex_alloc = false;
    int gtex_dirty = 7;
    uint64_t uid = 0;                // unique per volume of the process (a server's texture cache key)
    unsigned pyramid_version = 0;    // counts pyramid builds
    bool gather_tex_wanted() const { return params.gather_filter != 0 && params.precision != MRP_FP32; }
    // tensor-core predictor scratch
    TcScratch tc;
    // mrp_render_views
    mrpi::MultiViewBuffers mv;

    HitRecords records() const { return HitRecords{rec_count, rec_pix, rec_f, rec_cap}; }

    VolumeDev dev() const {
        VolumeDev d{};
        d.density = density;
        d.density_h = density_h;
        d.res = res;
        d.max_density = max_density;
        d.mips = mips;
        d.trs = trs;
        d.lut = lut;
        d.baked = baked;
        d.baked_res = bk_res;
        d.occ = occ;
        d.occ_shift = occ_shift;
        d.occ_res = occ_res;
        d.occ2 = occ2;
        d.occ2_res = occ2_res;
        d.scatter_rate = {params.scatter_rate[0], params.scatter_rate[1], params.scatter_rate[2]};
        d.tr_scale = params.tr_scale;
        d.sky = {params.sky[0] * params.env_exp, params.sky[1] * params.env_exp, params.sky[2] * params.env_exp};
        d.nee_mode = params.nee_mode;
        d.mip_occ = has_pyramid ? mip_occ : nullptr;
        d.mips_pad = has_pyramid ? mips_pad : nullptr;
        d.trs_pad = has_tr ? trs_pad : nullptr;
        d.mip_tr = has_tr ? mip_tr : nullptr;
        d.pad_pair = has_tr && has_pyramid ? pad_pair : nullptr;
        d.lut_dirs = has_lut ? lut + mrp::kLut * mrp::kLut : nullptr;
        d.hdri = hdri;
        d.hdri_w = hdri_w;
        d.hdri_h = hdri_h;
        d.env_exp = params.env_exp;
        d.has_bounds = has_bounds ? 1 : 0;
        if (gtex_alloc && gtex_dirty == 0 && gather_tex_wanted() && has_pyramid && has_tr && has_lut) {
            d.gmip0_tex = gmip0.tex;
            d.gtr0_tex = gtr0.tex;
            for (int l = 1; l < mrp::kGtexPairs; ++l) d.gpair_tex[l] = gpair[l].tex;
            d.glut_tex = glut.tex;
        }
        if (has_bounds) {
            // Density() at p reads base voxel floor((p + 0.5) R - 0.5) and the
            // next one: nonzero only for base voxels in [min - 1, max]; one
            // voxel of margin more on each side covers any rounding
            const float R = (float)res;
            d.nz_lo = {(nz_bounds[0] - 1.5f) / R - 0.5f, (nz_bounds[1] - 1.5f) / R - 0.5f,
                       (nz_bounds[2] - 1.5f) / R - 0.5f};
            d.nz_hi = {(nz_bounds[3] + 2.5f) / R - 0.5f, (nz_bounds[4] + 2.5f) / R - 0.5f,
                       (nz_bounds[5] + 2.5f) / R - 0.5f};
        }
        return d;
    }
};

namespace mrpi {
// The light of predictor launch `frame` when the volume has an environment
// map (core/volume.cu:494-509): L and C (light direction and colour) are
// replaced in place.  The launch's coin is the first uniform of Philox
// stream (kEnvLightStream, 0, 0, frame, seed) -- the reference calls rand().
void hdri_light(const mrp_volume* v, float coin, int n, float L[3], float C[3]);
inline void env_light_for_launch(const mrp_volume* v, uint32_t frame, uint32_t seed, float L[3], float C[3]) {
    uint32_t blk[4];
    mrp::philox(0, 0, frame, mrp::kEnvLightStream, 0u, seed ^ (mrp::kEnvLightStream * 0x9E3779B9u), blk);
    hdri_light(v, mrp::u01(blk[0]), v->hdri_light_n, L, C);
}
}  // namespace mrpi
