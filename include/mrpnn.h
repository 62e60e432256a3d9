/*
 * mrpnn.h -- C ABI of the MRPNN B200 render path (libmrpnn_b200.so).
 *
 * The reference exposes this path only as the C++ classes VolumeRender
 * (core/volume.hpp:45-155) and Camera (core/camera.hpp:29-43) over
 * process-global CUDA texture references.  This ABI carries the same
 * operations with opaque per-volume handles, plain pointers and sizes, and a
 * status code on every call; include/mrpnn_volume_render.hpp rebuilds the
 * reference's classes on top of it.  Each entry names the reference
 * interface it replaces.
 *
 * Conventions
 *   - Every call returns mrp_status; on failure mrp_last_error() holds a
 *     message (per calling thread).
 *   - 3D grids are res^3 floats, index (x*res + y)*res + z, z fastest
 *     (VolumeRender::SetData, core/volume.cu:1178-1180).
 *   - Buffers are caller-owned.  *_is_device = 0: host memory (pinned or
 *     pageable), copied inside the call; 1: device memory on the handle's
 *     device, used in place.
 *   - A volume handle owns one CUDA stream; calls on one handle are
 *     serialised by the caller, calls on different handles may run
 *     concurrently from different threads.  Calls return after the work
 *     they enqueue has completed unless documented otherwise.
 *   - Nothing here falls back to the CPU: without a usable sm_100 device
 *     mrp_init fails with MRP_ERR_NO_DEVICE.
 */
#ifndef MRPNN_H
#define MRPNN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum mrp_status {
    MRP_OK = 0,
    MRP_ERR_INVALID = 1,       /* bad argument                                 */
    MRP_ERR_NO_DEVICE = 2,     /* no CUDA device / not sm_100                  */
    MRP_ERR_CUDA = 3,          /* a CUDA runtime call failed                   */
    MRP_ERR_OOM = 4,           /* device allocation failed                     */
    MRP_ERR_NOT_READY = 5,     /* resource not built yet (e.g. no Update)      */
    MRP_ERR_UNSUPPORTED = 6,   /* e.g. RenderType RPNN (not compiled upstream) */
    MRP_ERR_IO = 7,            /* file could not be read / written             */
    MRP_ERR_BUDGET = 8,        /* serving: admission over the memory budget    */
    MRP_ERR_TIMEOUT = 9        /* serving: bounded wait expired                */
} mrp_status;

/* VolumeRender::RenderType (core/volume.hpp:98-100) */
typedef enum mrp_render_type { MRP_PT = 0, MRP_RPNN = 1, MRP_MRPNN = 2 } mrp_render_type;

/* MLP arithmetic of the predictor. FP32 is the drop-in (parity 1e-4 rel). */
typedef enum mrp_precision { MRP_FP32 = 0, MRP_BF16 = 1, MRP_FP8 = 2 } mrp_precision;

typedef struct mrp_volume mrp_volume;

/* Renderer settings that the reference keeps in __device__ globals
 * (core/render.cuh:10-18): VolumeRender::SetScatterRate, SetTrScale,
 * SetEnvExp.  sky is the constant environment radiance standing in for
 * SkyBox's HDRI (SetHDRI); bake_res is the NEE transmittance grid edge
 * (Update_CachedTR uses 768). */
typedef struct mrp_params {
    float scatter_rate[3];   /* default 1.001, 1.001, 1.001 */
    float tr_scale;          /* default 1                   */
    float sky[3];            /* default 0, 0, 0             */
    float env_exp;           /* default 1 (scales sky)      */
    int bake_res;            /* default 768                 */
    int bake_replicate_seeding; /* 1 (default): the reference's per-voxel estimates share one stream */
    mrp_precision precision; /* predictor MLP arithmetic, default MRP_FP32 */
    uint32_t seed;           /* RNG key of the LUT and bake streams, default 0 */
    int nee_mode;            /* PT next-event estimation: 0 (default) the baked
                                TR grid, as the reference; 1 one ratio-tracking
                                Tr() estimate per vertex (unbiased, no bake) */
    int tracer_filter;       /* the frame tracer's free-flight density fetch:
                                0 (default) software trilinear, fp32 weights in
                                the reference's float order; 1 the texture
                                unit's trilinear filter, as the reference's
                                tex3D (weights quantised to 1/256) */
    int gather_filter;       /* the stencil gather of the BF16 / FP8 forms
                                (fp16 features): 1 (default) the texture
                                unit's trilinear and bilinear filters on the
                                mip and TR levels and, for the light ray's
                                points, the HG-LUT, as the reference's own
                                tex3D / tex2D sampling in SetupInputData
                                (weights quantised to 1/256; the rotated
                                directions' LUT factor is read in software);
                                0 software filters with fp32 weights.  The
                                FP32 form always filters in software (the
                                oracle's features to ~1e-6). */
} mrp_params;

/* One camera: VolumeRender::Render(int2 size, ori, up, right, lightDir, rt,
 * g, alpha, lightColor, multiScatter, sampleNum) (core/volume.cu:487).  The
 * field of view follows |right| and |up| (unit vectors give 90 degrees). */
typedef struct mrp_view {
    int width, height;
    float ori[3], up[3], right[3];
    float light_dir[3], light_color[3];
    float alpha;             /* extinction scale                          */
    float g;                 /* Henyey-Greenstein asymmetry               */
    int multi_scatter;       /* PT bounce cap                             */
    int spp;                 /* PT samples per launch (reference: 32)     */
    uint32_t seed;           /* RNG key of the pixel streams              */
    int frame_offset;        /* launch index of the first launch          */
} mrp_view;

typedef struct mrp_volume_info {
    int res;
    float max_density;
    int has_pyramid, has_lut, has_tr, has_baked_tr;
    float lut_g, tr_alpha, tr_light[3];
    size_t device_bytes;
} mrp_volume_info;

/* Resource selector for mrp_volume_read (readback for checking). */
typedef enum mrp_resource {
    MRP_RES_DENSITY = 0, MRP_RES_MIP = 1, MRP_RES_TR = 2, MRP_RES_LUT = 3, MRP_RES_BAKED_TR = 4, MRP_RES_OCCUPANCY = 5
} mrp_resource;

/* -- library ---------------------------------------------------------------- */
/* cudaSetDevice + capability check; loads the model file if given (NULL:
 * the model file installed beside the library). */
mrp_status mrp_init(int device, const char* model_path);
const char* mrp_last_error(void);
const char* mrp_version(void);
/* Number of CUDA allocation and free calls (device, stream-ordered and
 * pinned host) the library has made since it was loaded.  No counterpart in
 * the reference; a diagnostic that lets a caller check that an entry point
 * which promises not to allocate (mrp_predict_features_noalloc) made no such
 * call.  Needs no device. */
unsigned long long mrp_debug_alloc_calls(void);
/* Replaces the network weights from a model file (format: mrpnn_b200/data/
 * make_model.py).  The reference bakes them into __constant__ arrays
 * (core/NNWeight.cuh, core/radiancePredict.cu:299). */
mrp_status mrp_load_model(const char* path);
void mrp_default_params(mrp_params* p);

/* -- volume lifecycle --------------------------------------------------------- */
/* VolumeRender(int resolution) (core/volume.cu:948-957); allocates exactly
 * res^3 floats instead of the reference's fixed 1024^3 array. */
mrp_status mrp_volume_create(int res, mrp_volume** out);
/* Storage type of the density grid.  FP16 halves the grid's HBM (a 1024^3
 * volume: 2 GiB instead of 4); values are rounded to nearest on the way in
 * (set_data, fill, generate_fbm) and widened exactly on every read, so an
 * FP16 volume renders exactly as an FP32 volume holding the rounded values.
 * The pyramid, TR levels, LUT and baked grid stay fp32.  The reference keeps
 * the grid as float only (core/volume.hpp:47, datas). */
typedef enum mrp_storage { MRP_STORAGE_FP32 = 0, MRP_STORAGE_FP16 = 1 } mrp_storage;
mrp_status mrp_volume_create_ex(int res, mrp_storage storage, mrp_volume** out);
/* ~VolumeRender (core/volume.cu:1151-1176) */
mrp_status mrp_volume_destroy(mrp_volume* v);
/* VolumeRender::SetDatas / SetData storage (core/volume.cu:1178-1184):
 * copies a full res^3 grid. */
mrp_status mrp_volume_set_data(mrp_volume* v, const float* data, int res, int is_device);
/* SetDatas(FillFunc) through ParallelFill (core/omp.cpp:4-18): fn(x,y,z,u,v,w)
 * with u = (x+0.5)/res, evaluated on host threads. */
typedef float (*mrp_fill_fn)(int x, int y, int z, float u, float v, float w, void* user);
mrp_status mrp_volume_fill(mrp_volume* v, mrp_fill_fn fn, void* user);
/* Synthetic fBm cloud generated on the device (benchmark volumes). */
mrp_status mrp_volume_generate_fbm(mrp_volume* v, uint32_t seed, float base_freq, int octaves, float gain);
/* VolumeRender::Update(process_mips) (core/volume.cu:1443-1531): computes the
 * majorant (max density, which the reference leaves at 1e-5), the 9-level
 * pyramid (256>>m) and the occupancy bricks, on the device. */
mrp_status mrp_volume_update(mrp_volume* v, int process_mips);
/* Overrides the majorant (the reference's max_density field). */
mrp_status mrp_volume_set_max_density(mrp_volume* v, float max_density);
mrp_status mrp_volume_get_info(const mrp_volume* v, mrp_volume_info* info);
mrp_status mrp_set_params(mrp_volume* v, const mrp_params* p);
mrp_status mrp_get_params(const mrp_volume* v, mrp_params* p);
/* Copies a resource (level: mip / TR level) to dst; returns its float count
 * in *count when dst is NULL. */
mrp_status mrp_volume_read(mrp_volume* v, mrp_resource which, int level, float* dst, size_t* count, int dst_is_device);

/* -- environment map: VolumeRender::SetHDRI(path) (core/volume.cu:1696-1728) -- */
/* Reads a Radiance RGBE .hdr file as the reference's loader does
 * (core/hdr_loader.h): width x height RGBA floats, rows top to bottom,
 * (m + 0.5) 2^(e - 136) per channel, alpha 0.  Host only.  rgba == NULL:
 * only the size is returned. */
mrp_status mrp_hdri_file_read(const char* path, int* width, int* height, float* rgba, size_t rgba_floats);
/* Sets the volume's equirect environment map (host RGBA floats, width x
 * height; NULL clears it: the constant sky of mrp_params.sky returns).
 * SkyBox then samples it (bilinear, wrap addressing) times env_exp for every
 * ray that leaves the volume, in the tracer, the predictor's missed pixels,
 * the batch-ray APIs and the viewer frame; and each predictor launch of
 * mrp_render / mrp_render_start, each viewer frame and each served request
 * is lit either by the map (from its Roberts2 direction, with probability
 * 4 env_exp / (4 env_exp + max light colour)) or by the sun with its colour
 * divided by 1 - that probability, as the reference's Render does
 * (core/volume.cu:494-509); the coin is Philox stream (6, 0, 0, frame, seed)
 * instead of rand().  mrp_render_views keeps the views' own light.  Not
 * while requests on this volume are in flight in a server. */
mrp_status mrp_volume_set_hdri(mrp_volume* v, const float* rgba, int width, int height);
/* mrp_hdri_file_read + mrp_volume_set_hdri. */
mrp_status mrp_volume_load_hdri(mrp_volume* v, const char* path);

/* VolumeRender::GetHGLut(cos, angle) (core/volume.cu:1424-1442): the HG
 * lookup table (512 x 512, row = cone angle, column = cos theta, as
 * mrp_volume_read(MRP_RES_LUT) returns it) read at (cos, angle) with the
 * reference's host arithmetic, quirks included (the two texels of a row are
 * blended with the row fraction, the two rows with the column fraction).
 * Host only (no device needed). */
mrp_status mrp_hg_lut_lookup(const float* lut, float cos_theta, float angle, float* out);

/* -- volume files: VolumeRender(string path, bool cacheTR) / LoadData
 * (core/volume.cu:970-1149) --------------------------------------------------------- */
/* .bin (int32 R, R^3 float32, z fastest), .txt (R then R^3 floats) or .vox
 * (256^3 integers x 64/255); a path without a .bin suffix reads path + ".bin"
 * when that cache exists.  Host only (no device needed).  dst == NULL: only
 * *res is returned. */
mrp_status mrp_volume_file_read(const char* path, int* res, float* dst, size_t dst_floats);
/* Writes the .bin format (the reference's cache file). */
mrp_status mrp_volume_file_write_bin(const char* path, const float* data, int res);
/* Reads a volume file into a new handle and runs mrp_volume_update.  The
 * reference's four datasets (path containing CLOUD0, CLOUD1, MODEL0, MODEL1)
 * keep its hard-coded majorants; write_cache = 1 writes path + ".bin" after
 * parsing a .txt / .vox file, as LoadData does. */
mrp_status mrp_volume_load(const char* path, int write_cache, mrp_volume** out);

/* -- per-render caches ------------------------------------------------------------ */
/* VolumeRender::UpdateHGLut(g) (core/volume.cu:1401-1423), cached on g. */
mrp_status mrp_update_hg_lut(mrp_volume* v, float g);
/* VolumeRender::Update_TR(lightDir, alpha) (core/volume.cu:1589-1667),
 * cached on (lightDir, alpha). */
mrp_status mrp_update_tr(mrp_volume* v, const float light_dir[3], float alpha);
/* VolumeRender::Update_CachedTR(lightDir, alpha) (core/volume.cu:1669-1696),
 * cached on (lightDir, alpha, bake_res). */
mrp_status mrp_update_baked_tr(mrp_volume* v, const float light_dir[3], float alpha);

/* -- rendering ---------------------------------------------------------------------- */
/* VolumeRender::Render(...) -> vector<float4> (core/volume.cu:487-548):
 * sample_num launches with the running mean of RenderCamera; out holds
 * width*height float4 (RGB, A = coverage for PT / hit distance for MRPNN). */
mrp_status mrp_render(mrp_volume* v, const mrp_view* view, mrp_render_type type, int sample_num, float* out_rgba,
                      int out_is_device);
/* mrp_render that returns once the render is queued (no counterpart in the
 * reference, whose Render synchronises per launch, core/volume.cu:536): the
 * result is copied to out_rgba on a second stream while the next started
 * render computes, so a frame loop's copies back to the host overlap the
 * device work.  Two results alternate between two device buffers; a third
 * start waits on the device for the first one's copy.  out_rgba must stay
 * valid and untouched until mrp_render_wait returns; host buffers must be
 * pinned for the copy to overlap (pageable ones make the start synchronous).
 * Any other call on the volume that uses the result buffers (mrp_render,
 * the interactive frame, a render that needs larger buffers) first waits. */
mrp_status mrp_render_start(mrp_volume* v, const mrp_view* view, mrp_render_type type, int sample_num, float* out_rgba,
                            int out_is_device);
/* keep = 0: blocks until every started render of v is in its output buffer,
 * and reports a tensor-core wait that timed out in any of them
 * (MRP_ERR_TIMEOUT).  keep = 1: until every one but the newest is -- a frame
 * loop starts frame k, waits with keep = 1 and reads frame k - 1 while frame
 * k computes. */
mrp_status mrp_render_wait(mrp_volume* v, int keep);
/* One launch of mrp_render (output discarded) that also counts its work:
 * MRPNN: [0] march steps, [1] density fetches (steps not skipped by the
 * occupancy bricks), [2] stencil points gathered, [3] hit pixels;
 * PT: [0] bounces, [1] free-flight density fetches, [2] NEE transmittance
 * lookups, [3] samples traced.  For roofline accounting; not timed. */
mrp_status mrp_render_counters(mrp_volume* v, const mrp_view* view, mrp_render_type type, unsigned long long counters[4]);
/* Device time of the kernels of the last mrp_render on this handle (ms;
 * -1 when it ran more than one launch -- see mrp_last_render_stages). */
mrp_status mrp_last_render_ms(const mrp_volume* v, float* ms);
/* Device time of the stages of the last launch of the last mrp_render (ms):
 * MRPNN = first hit + bases, stencil gather, network; PT = paths, resolve, 0. */
mrp_status mrp_last_render_stages(const mrp_volume* v, float ms[3]);

/* n (1..64) MRPNN views of one volume in one call, the network of all views
 * in one batched persistent launch.  No counterpart in the reference (its
 * data generator calls Render once per camera, dataGen.cu:246-328).  The
 * views share light_dir, alpha and g (one TR / LUT state); each image equals
 * mrp_render of that view with sample_num 1.  outs[i]: width*height*4
 * floats.  Stage times (mrp_last_render_stages): hit + gather of all views,
 * network, result copies. */
mrp_status mrp_render_views(mrp_volume* v, const mrp_view* views, int n, float* const* outs, int outs_are_device);

/* -- interactive frames: VolumeRender::Render(float3*, Histogram*, unsigned*, ...)
 * (core/volume.cu:550-628) ------------------------------------------------------------ */
/* Histogram (core/volume.hpp:12-19): 10 bins per channel of L / (L + 1), the
 * sample count and running means of the luminance and its square. */
typedef struct mrp_histogram {
    float bin[30];
    float total, x2, x;
} mrp_histogram;
/* One viewer frame.  PT: one sample per (checkerboard-selected) pixel into
 * the running mean `target` and the histograms, then Denoise (histogram-
 * weighted 11 x 11 filter when denoise != 0 and the pixel's variance > 0.01;
 * checkerboard fill on frame 0); MRPNN: target = the prediction at the
 * selected pixels, then ReprojectionDenoise.  Both end in exposure, tone
 * (0 none, 1 Gamma, 2 ACES) and an RGBA8 pack 0xff000000 | r<<16 | g<<8 | b.
 * frame_num is the reference's frameNum (running-mean index; halved with
 * checkerboard), flip its checkerboard parity; view->frame_offset keys the
 * RNG.  target (w*h*3 floats) and histo (w*h) are device buffers the caller
 * owns and keeps between frames (zero them before frame 0); rgba8 (w*h) is
 * device or host memory.  Images follow the interactive kernel's framing
 * (v = (row + r) / H). */
mrp_status mrp_render_interactive(mrp_volume* v, const mrp_view* view, mrp_render_type type, int frame_num,
                                  int checkerboard, int flip, int tone, int denoise, float exposure, float* target,
                                  mrp_histogram* histo, uint32_t* rgba8, int rgba8_is_device);

/* -- batch ray APIs (core/volume.cu:405-479, 710-834) ---------------------------------
 * ori / dir / light_dirs: [n][3]; outputs [n][3]; is_device covers inputs and
 * output alike. */
/* VolumeRender::GetRadiances: CalculateRadiance (PT, sample_num samples, NEE
 * as mrp_params.nee_mode) or NNPredict<MRPNN> (network precision as the
 * volume's params) for each ray; RGB only. */
mrp_status mrp_get_radiances(mrp_volume* v, const float* ori, const float* dir, int n, const float light_dir[3],
                             const float light_color[3], float alpha, int multi_scatter, float g, int sample_num,
                             mrp_render_type type, float* out3, int is_device);
/* VolumeRender::GetSamples (GetSample, core/render.cuh:615-655), the training
 * data generator: per task alpha, origin in the medium, view direction,
 * light direction, g and scatter rate. */
mrp_status mrp_get_samples(mrp_volume* v, const float* alpha, const float* ori, const float* dir,
                           const float* light_dirs, const float* g, const float* scatter, int n,
                           const float light_color[3], int multi_scatter, int sample_num, uint32_t seed, float* out3,
                           int is_device);
/* VolumeRender::GetTrs (ShadowTerm_TRs, core/render.cuh:668-680): light
 * colour x pi x mean of Tr() x HG toward the light. */
mrp_status mrp_get_trs(mrp_volume* v, float alpha, const float* ori, const float* dir, int n,
                       const float light_dir[3], const float light_color[3], float g, int sample_num, uint32_t seed,
                       float* out3, int is_device);

/* VolumeRender::GatherData (core/volume.cu:630-700 -> GatherSamples ->
 * NNGatherSamples, core/render.cuh:1006-1142): the input of the tile network
 * for a view->width x view->height grid of 8 x 8-pixel tiles, sub-pixel offset
 * (px, py) in eighths of a tile.  out [tiles][773]: X_Val[192],
 * X_Val_Hg[192], X_Val_Sub[192] (SetupInputData2 of 16 depth samples), 5
 * angle / depth-gradient terms, 192 t-grid values; a tile whose 64 rays all
 * miss has out[0] = -1000 (the rest zero apart from its t-grid). */
mrp_status mrp_gather_tiles(mrp_volume* v, const mrp_view* view, int px, int py, float* out, int is_device);

/* -- parity entry points (pieces of the path) ---------------------------------------- */
/* RadiancePredictInternal (core/radiancePredict.cu:301-422) on n feature
 * sets: feat [n][576] = X_Val[192], X_Val_Sub[192], X_Val_Hg[192]; gamma [n];
 * out [n][3]. */
mrp_status mrp_predict_features(const float* feat, const float* gamma, float g, const float scatter_rate[3], int n,
                                float* out3, mrp_precision precision, int is_device);
/* No counterpart in the reference.  mrp_predict_features for host buffers
 * that allocates nothing.  It is for callers that must not allocate while
 * they render: a frame loop that cannot afford the device-wide
 * synchronisation cudaFree implies, or a process whose memory pool
 * (PyTorch's caching allocator, say) already holds the HBM, so that a
 * cudaMalloc could fail in the middle of a frame.  The device copies of feat
 * and gamma, the output, and the tensor-core network's tile counter and error
 * flag live in one fixed array in the library's device image,
 * MRP_NOALLOC_SCRATCH_BYTES (about 4.5 MiB), which every GPU that loads the
 * library holds until the process exits.
 *   - n <= MRP_NOALLOC_MAX_POINTS; a larger n returns MRP_ERR_INVALID and
 *     does nothing -- split the batch.
 *   - The array keeps the last call's contents.  The tile counter and the
 *     error flag must start at zero, and each call clears both on its stream
 *     before it launches; the feature area needs no clearing.
 *   - The first call on a device looks the array's device address up
 *     (cudaGetSymbolAddress, which may load the module); make that first call
 *     before any stream capture begins.
 *   - All calls share the array, so calls that overlapped on the GPU would
 *     race on it.  The library holds its lock for the whole call and returns
 *     only after its stream has drained, so calls from several host threads
 *     run one after another. */
#define MRP_NOALLOC_MAX_POINTS 2048
#define MRP_NOALLOC_SCRATCH_BYTES (256 + (size_t)MRP_NOALLOC_MAX_POINTS * (576 + 1 + 3) * 4)
mrp_status mrp_predict_features_noalloc(const float* feat, const float* gamma, float g, const float scatter_rate[3],
                                        int n, float* out3, mrp_precision precision);
/* SetupInputData (core/radiancePredict.cu:427-485) for n points: pos [n][3],
 * bases [n][12] = XMain, YMain, ZMain, LXMain; feat [n][576], gamma [n]. */
mrp_status mrp_gather_features(mrp_volume* v, const float* pos, const float* bases, const float light_dir[3], float g,
                               float alpha, int n, float* feat, float* gamma, int is_device);
/* GetSamplePoint (core/render.cuh:436-462) for n rays: hit4 [n][4] =
 * (x, y, z, 1 if hit). */
mrp_status mrp_first_hit(mrp_volume* v, const float* ori, const float* dir, float alpha, int n, float* hit4,
                         int is_device);

/* Tensor-core check: D[128][n] = A[128][k] * B[n][k]^T (row-major fp32 in,
 * fp32 out) with A and B rounded to BF16 (fp8 = 0) or E4M3 (fp8 = 1) and
 * accumulated in FP32 by one tcgen05.mma chain -- the operand layout and
 * descriptors of the tensor-core MLP.  n: 16..128 step 16; k: multiple of 16
 * (32 for E4M3) up to 128. */
mrp_status mrp_tc_gemm_check(int fp8, const float* A, const float* B, int n, int k, float* D);

/* Measured rate (GB/s) at which the SMs return cached 8-byte read-only loads
 * (every CTA reads its own 16 KiB window, eight loads in flight per thread):
 * the ceiling of the stencil gather's texel reads, which hit L1.  No
 * counterpart in the reference (a measurement of this GPU). */
mrp_status mrp_measure_l1_rate(float* gbs);
/* The rate (GB/s) at which this GPU's SMs read 16-byte words that bypass L1
 * from a 64 MiB buffer resident in L2: the ceiling the bench states the
 * tracer's L2-resident density reads against.  No counterpart in the
 * reference; allocates and frees its buffer. */
mrp_status mrp_measure_l2_rate(float* gbs);

/* One MRPNN launch of mrp_render (launch index view->frame_offset, no
 * running mean) that also returns the intermediates of NNPredict per pixel:
 * aux [w*h][20] = hit x, y, z, hit flag, gamma, XMain, YMain, ZMain, LXMain
 * (GetSamplePoint, GetMatrixFromNormal, core/render.cuh:808-843) and feat
 * [w*h][576] (SetupInputData's features; zero where no hit).  It runs the
 * volume's precision: with MRP_FP32 the fp32 features and network, with
 * MRP_BF16 / MRP_FP8 the fp16 features (returned widened to float) and the
 * tensor-core network, so rgba equals mrp_render's image of that launch. */
mrp_status mrp_render_predict_debug(mrp_volume* v, const mrp_view* view, float* rgba, float* aux, float* feat,
                                    int is_device);

/* -- serving --------------------------------------------------------------------------
 * The reference renders one frame per synchronous Render call
 * (core/volume.cu:487-548); its viewer (core/GUI.hpp:1002-1030) and data
 * generator (dataGen.cu:246-328) loop over it.  A server keeps any number of
 * resident volumes (ordinary mrp_volume handles after mrp_volume_update) and
 * renders MRPNN requests on them with continuous batching: a worker thread
 * admits requests into slots while slots and the memory budget allow; each
 * admitted request builds its own TR mips for its light and alpha and runs
 * the first hit and the stencil gather on its slot's stream, overlapping the
 * requests already on the device; the network of every request whose
 * features are ready runs in one batched persistent launch; results go to
 * the caller's buffer.  Each result equals mrp_render of the same view with
 * sample_num 1 (same kernels, same per-pixel streams).
 * Volumes must not be changed (set_data / update / params) while requests on
 * them are pending. */
typedef struct mrp_server mrp_server;
typedef struct mrp_serve_config {
    size_t memory_budget;    /* device bytes for request slots and LUTs (default 120 GB) */
    int max_slots;           /* requests on the device at once, 1..64 (default 16) */
    mrp_precision precision; /* network arithmetic (default MRP_BF16)              */
    size_t slot_pixels;      /* size every slot for this many pixels at open, so
                                admission never allocates (default 0: slots grow
                                on demand, stream-ordered, and keep their size) */
} mrp_serve_config;
typedef struct mrp_request {
    mrp_volume* volume;      /* resident volume (pyramid built)                    */
    mrp_view view;           /* camera, light, alpha, g, seed, frame_offset        */
    float* out_rgba;         /* width*height*4 floats, as mrp_render writes them   */
    int out_is_device;       /* 0: host memory (pinned or pageable), 1: device     */
} mrp_request;
/* Milliseconds since mrp_serve_open of each step of one request. */
typedef struct mrp_request_timing {
    double submit_ms, admit_ms, features_ms, network_ms, done_ms;
} mrp_request_timing;
typedef struct mrp_serve_stats {
    unsigned long long submitted, completed, failed, batches, batched_requests;
    int max_batch;           /* most requests in one network launch               */
    size_t bytes_in_use, peak_bytes;
} mrp_serve_stats;
void mrp_serve_default_config(mrp_serve_config* cfg);
mrp_status mrp_serve_open(const mrp_serve_config* cfg, mrp_server** out);
/* Queues a request; returns at once with its ticket.  A request larger than
 * the whole budget fails with MRP_ERR_BUDGET here. */
mrp_status mrp_serve_submit(mrp_server* s, const mrp_request* req, uint64_t* ticket);
/* Waits up to wait_ms (0: poll; < 0: until done) for a ticket.  *done = 1
 * when the result is in the caller's buffer; the return value is then the
 * request's own status and the ticket is released.  *done = 0: still
 * running, MRP_OK. */
mrp_status mrp_serve_poll(mrp_server* s, uint64_t ticket, int wait_ms, int* done, mrp_request_timing* timing);
mrp_status mrp_serve_stats_get(mrp_server* s, mrp_serve_stats* stats);
/* Finishes every submitted request, then stops the worker and frees the
 * server's device memory. */
mrp_status mrp_serve_close(mrp_server* s);

#ifdef __cplusplus
}
#endif
#endif /* MRPNN_H */
