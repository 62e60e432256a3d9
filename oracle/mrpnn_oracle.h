/*
 * mrpnn_oracle.h -- CPU restatement of the MRPNN render path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * product in mrpnn_b200/.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  It is never
 * linked into, called by, or used as a fallback for the product path.
 *
 * Parity pin: the pieces below that have a host-compilable counterpart in the
 * reference (the MLP RadiancePredictInternal, SetupInputData, the stencil
 * tables, HenyeyGreenstein / ray-box / sampling maths, DeterminateEstimatedHit,
 * GetMatrixFromNormal, DeterminateNextVertex, CalculateRadiance and Tr) are
 * checked against the reference's own sources compiled on the CPU by the
 * recipe in oracle/ref/ (outputs into oracle/_ref/), and against golden
 * vectors generated from that build (tests/golden/).  The volume builders --
 * the pyramid of Update, Fill_TR, Fill_Hg, GetHGLut and Fill_BakeTR -- are
 * pinned the same way to core/volume.cu compiled on the CPU by that recipe
 * (kernel launches rewritten to a host launcher, CUDA arrays as host memory).
 *
 * All float arithmetic is compiled with -ffp-contract=off so that the order
 * of roundings is the one written here; the CUDA kernels use the same order
 * with non-contracting intrinsics.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Scene resources, host memory.  Layout of every 3D grid: index
 * (x*R + y)*R + z, z fastest (core/volume.cu:1179). */
typedef struct orc_scene {
    const float* density;   /* full-resolution grid, res^3                      */
    int res;                /* its resolution ("Resolution", core/render.cuh:10) */
    float max_density;      /* majorant density ("maxDensity")                  */
    const float* mips;      /* 9 levels, level m is (256>>m)^3, concatenated    */
    const float* tr_mips;   /* 8 levels, level i is (128>>i)^3, concatenated    */
    const float* hg_lut;    /* 512x512, index v_row*512 + u_col                 */
    const float* baked_tr;  /* NEE transmittance grid used by the tracer; NULL:
                               one Tr() estimate per vertex instead (unbiased)   */
    int baked_res;
    float scatter_rate[3];  /* "scatter_rate" (core/render.cuh:17)              */
    float tr_scale;         /* "tr_scale" (core/render.cuh:16)                  */
    float sky[3];           /* constant environment radiance, used when no map  */
    const float* hdri;      /* equirect environment map, RGBA float rows of
                               hdri_w texels (SetHDRI); NULL: constant sky      */
    int hdri_w, hdri_h;
    float env_exp;          /* "enviroment_exp" (core/render.cuh:15), scales the map */
} orc_scene;

/* One camera launch.  Mirrors RenderCamera's arguments (core/volume.cu:199). */
typedef struct orc_view {
    int width, height;
    float ori[3], up[3], right[3];
    float light_dir[3], light_color[3];
    float alpha, g;
    int multi_scatter;      /* tracer bounce cap                                 */
    int spp;                /* tracer samples per launch (reference: 32)         */
    uint32_t seed;          /* RNG key                                           */
    int frame;              /* launch index ("frameNum"/"randNum")               */
} orc_view;

/* ---- RNG: Philox-4x32-10 (Salmon et al., SC'11) ------------------------- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* n-th uniform of stream (kind, id, sub, frame, seed): word n % 4 of
 * Philox(counter = (n / 4, sub, frame, kind), key = (id, seed ^ kind * 0x9E3779B9)),
 * mapped to (0, 1) as the device streams do. */
float orc_stream_uniform(uint32_t kind, uint32_t id, uint32_t sub, uint32_t frame,
                         uint32_t seed, uint32_t n);

/* ---- model file ---------------------------------------------------------- */
int  orc_load_model(const char* path);          /* 0 on success */
int  orc_model_tensor(const char* name, const float** data, int* count);

/* ---- synthetic volumes ----------------------------------------------------- */
float orc_fbm_voxel(int R, int x, int y, int z, uint32_t seed, float base_freq,
                    int octaves, float gain);
void  orc_fbm_volume(float* out, int R, uint32_t seed, float base_freq, int octaves,
                     float gain);
float orc_max_density(const float* d, int64_t n);

/* ---- volume resources ----------------------------------------------------- */
void orc_build_pyramid(const float* data, int R, float* mips_out);
void orc_tr_mip_level(const float* mips, int level, float alpha, const float light_dir[3],
                      float* out);
void orc_hg_lut_texels(float g, uint32_t seed, const int* texels, int n, float* out);
void orc_baked_tr(const orc_scene* s, float alpha, const float light_dir[3], int bake_res,
                  uint32_t seed, int replicate_reference_seeding, const int64_t* voxels,
                  int64_t n, float* out);
float orc_tr(const orc_scene* s, const float pos[3], const float dir[3], float dis,
             float alpha, uint32_t stream_id, uint32_t sub, uint32_t frame, uint32_t seed,
             uint32_t kind);

/* ---- stencil tables --------------------------------------------------------- */
void orc_stencil_tables(float* offset, int* layer, int* type, int* localindex, float* lut_v);

/* ---- maths --------------------------------------------------------------- */
float orc_hg(float cosv, float g);
void  orc_sample_hg(float e0, float e1, const float v[3], float g, float out[3]);
float orc_ray_box_offset(const float p[3], const float d[3]);
float orc_ray_box_distance(const float p[3], const float d[3]);
float orc_sample_density(const float* grid, int n, const float pos[3], int clamp_mode);
float orc_sample_lut(const float* lut, float u, float v);

/* ---- predictor pieces ----------------------------------------------------- */
/* Camera ray of pixel (row, col) for launch `frame`: dir (normalized), plus the
 * jitter draws.  RenderCamera, core/volume.cu:201-216. */
void orc_camera_ray(const orc_view* v, int row, int col, float dir_out[3]);
/* GetSamplePoint/DeterminateEstimatedHit(float&): returns 1 if a hit. */
int  orc_first_hit(const orc_scene* s, const float ori[3], const float dir[3], float alpha,
                   float hit_out[3]);
/* GetMatrixFromNormal for the pixel stream at draw cursor *cursor. */
void orc_basis(const float v[3], float spread, uint32_t id, uint32_t sub, uint32_t frame,
               uint32_t seed, uint32_t* cursor, float out9[9]);
/* SetupInputData, core/radiancePredict.cu:427-485.  feat: [3][192] = X_Val,
 * X_Val_Sub, X_Val_Hg (the channel order the MLP pools them in). */
void orc_setup_input(const orc_scene* s, int active, const float pos[3], const float X[3],
                     const float Y[3], const float Z[3], const float LX[3],
                     const float light[3], float g, float alpha, float* feat576,
                     float* gamma_out);
/* RadiancePredictInternal, core/radiancePredict.cu:301-422, per pixel. */
void orc_mlp_f32(const float* feat, const float* gamma, float g, const float sr[3], int n,
                 float* out3);
void orc_mlp_f64(const float* feat, const float* gamma, float g, const float sr[3], int n,
                 double* out3);
/* NNPredict<MRPNN> for pixels of one launch (no running mean): rgba out. */
void orc_predict_pixels(const orc_scene* s, const orc_view* v, const int* pixels, int n,
                        float* rgba_out, float* feat_out, float* gamma_out, float* hit_out);
/* CalculateRadiance for pixels of one launch: per-pixel mean over v->spp
 * samples (float4, as the reference) plus FP64 sums of L and L^2 per channel. */
void orc_trace_pixels(const orc_scene* s, const orc_view* v, const int* pixels, int n,
                      float* rgba_out, double* sum3, double* sumsq3);
/* GetRadiances (PT) for explicit rays ori/dir [n][3]: FP64 sums over v->spp. */
void orc_trace_rays(const orc_scene* s, const orc_view* v, const float* ori, const float* dir, int n, double* sum3,
                    double* sumsq3);
/* GetSamples: per task alpha, ori, dir, light dir, g, scatter; out [n][3]. */
void orc_get_samples(const orc_scene* s, const float* alpha, const float* ori, const float* dir, const float* ldir,
                     const float* g, const float* scatter, int n, const float lc[3], int multi_scatter, int spp,
                     uint32_t seed, float* out3);
/* Interactive frame: PT sample + running mean + histograms at the
 * (checkerboard-)selected pixels (histo: 33 floats per pixel: bin[30],
 * total, x2, x), and the Denoise / ReprojectionDenoise + tone + RGBA8 pass. */
void orc_frame_pt(const orc_scene* s, const orc_view* v, int fnum, int checker, int flip, float* target,
                  float* histo);
void orc_frame_finish(const float* target, float* histo, int W, int H, int frame_num, int flip, int predict,
                      int denoise, float exposure, int tone, uint32_t* rgba8);
/* GatherData (tile features of the tile network): v->width x v->height tiles,
 * sub-pixel offset (px, py) in 1/8 tile; out [tiles][773]. */
void orc_gather_tiles(const orc_scene* s, const orc_view* v, int px, int py, float* out);
/* GetTrs: ShadowTerm_TRs per task; out [n][3]. */
void orc_get_trs(const orc_scene* s, float alpha, const float* ori, const float* dir, int n, const float L[3],
                 const float lc[3], float g, int spp, uint32_t seed, float* out3);
/* The light of one predictor launch with an environment map
 * (core/volume.cu:494-509): L, C replaced in place; coin in [0, 1) stands in
 * for rand() / RAND_MAX, n is the Roberts2 index (rand_cpu).  The pieces
 * Roberts2 (core/vector.cu:179-183), UniformSampleSphere (:195-205) and
 * Image_host::Sample (core/volume.hpp:24-42) are exported for the pins. */
void orc_env_light(const orc_scene* s, float coin, int n, float L[3], float C[3]);
void orc_roberts2(int n, float out[3]);
void orc_uniform_sample_sphere(float ex, float ey, float out[3]);
void orc_image_sample(const float* rgba, int sx, int sy, float u, float v, float out[3]);

#ifdef __cplusplus
}
#endif
