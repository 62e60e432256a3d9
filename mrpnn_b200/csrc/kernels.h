// kernels.h -- launch entry points of the MRPNN B200 kernels (host side).
#pragma once
#include "common.cuh"
#include "dev_alloc.h"

namespace mrp {

// volume_kernels.cu
// The density grid's builders take fp32 or fp16 storage (VolumeDev::density
// or density_h); everything derived from it (pyramid, TR, LUT) is fp32.
cudaError_t launch_fbm(float* out, int R, uint32_t seed, float base_freq, int octaves, float gain, int sms,
                       cudaStream_t s);
cudaError_t launch_fbm(__half* out, int R, uint32_t seed, float base_freq, int octaves, float gain, int sms,
                       cudaStream_t s);
cudaError_t launch_narrow(const float* in, size_t n, __half* out, int sms, cudaStream_t s);
cudaError_t launch_widen(const __half* in, size_t n, float* out, int sms, cudaStream_t s);
cudaError_t launch_resample(float* out, int res, const float* src, int src_res, int sms, cudaStream_t s);
cudaError_t launch_resample(float* out, int res, const __half* src, int src_res, int sms, cudaStream_t s);
cudaError_t launch_max_density(const float* d, size_t n, int* out_bits, int sms, cudaStream_t s);
cudaError_t launch_max_density(const __half* d, size_t n, int* out_bits, int sms, cudaStream_t s);
cudaError_t launch_occupancy(const float* d, int R, int shift, int nb, uint8_t* occ, int sms, cudaStream_t s);
cudaError_t launch_occupancy(const __half* d, int R, int shift, int nb, uint8_t* occ, int sms, cudaStream_t s);
// Coarse bricks (edge 4 bricks) of an occupancy grid of nb^3 bricks: (nb+3)/4 per axis.
cudaError_t launch_occupancy_coarse(const uint8_t* occ, int nb, uint8_t* coarse, int sms, cudaStream_t s);
// VolumeDev::pad_pair from the padded mips and TR levels (kPadLevelFloats pairs).
cudaError_t launch_pair_padded(const float* mips_pad, const float* trs_pad, float2* out, cudaStream_t s);
// VolumeDev::mip_tr from the pyramid and the TR levels (mip_tr_offset(5) pairs).
cudaError_t launch_interleave_mip_tr(const float* mips, const float* trs, float2* out, int sms, cudaStream_t s);
// Padded copies (pad_offset layout, kPadLevelFloats floats) of three levels
// of edge 8, 4, 2; clamp: TR-level addressing, else border (density mips).
cudaError_t launch_pad_levels(const float* l8, const float* l4, const float* l2, bool clamp, float* out,
                              cudaStream_t s);
// Index bounds of the nonzero voxels: out6 = {min x, min y, min z, max x,
// max y, max z}, which must start at {R, R, R, -1, -1, -1}.
cudaError_t launch_nonzero_bounds(const float* d, int R, int* out6, int sms, cudaStream_t s);
cudaError_t launch_nonzero_bounds(const __half* d, int R, int* out6, int sms, cudaStream_t s);
cudaError_t launch_tr_level(float* out, int res, const float* src, const uint8_t* src_occ, float alpha, const float L[3], int sms,
                            cudaStream_t s);
cudaError_t set_halton_permutations(const uint32_t perm[28]);
cudaError_t launch_hg_lut(float* lut, float g, uint32_t seed, cudaStream_t s);
cudaError_t launch_baked_tr(float* out, const VolumeDev& v, int bake_res, float alpha, const float L[3], uint32_t seed,
                            int replicate, int sms, cudaStream_t s);

// predictor_kernels.cu
struct StencilTables {
    float offset[192];
    int layer[192];
    float lut_v[192];
    float dirs[160 * 3];
};
cudaError_t set_stencil_tables(const StencilTables& t);
// lut_dirs (160 floats) of the LUT at lut (the table VolumeDev::lut_dirs
// points at), after the LUT is built on the same stream.
cudaError_t launch_lut_dirs(const float* lut, float* out, cudaStream_t s);
// features: [n][576] (X_Val, X_Val_Sub, X_Val_Hg), gamma [n]
cudaError_t launch_gather(const VolumeDev& v, const float* pos, const float* bases, const float* light, float g,
                          float alpha, int n, float* feat, float* gamma, cudaStream_t s);
cudaError_t launch_mlp_fp32(const float* weights, const float* feat, const float* gamma, float g, const float sr[3],
                            int n, float* out3, cudaStream_t s);
cudaError_t launch_first_hit(const VolumeDev& v, const float* ori, const float* dir, float alpha, float pass_rate, int n,
                             float* hit4, cudaStream_t s);
// Staged predictor (one launch of RenderCamera<true, MRPNN>, running mean
// into accum with weight 1/(1+mean_k)):
//   launch_hit         ray + first hit + bases, compact list of hit pixels
//   launch_gather_rec  stencil features of the hit pixels (tiled layout)
//   launch_mlp_rec_*   network on the features, result at each pixel
struct HitRecords {
    int* count;     // [0] number of records, [1] the march's work counter (device; launch_hit zeroes both)
    int* pix;       // [cap] pixel index of each record
    float* f;       // [16][cap]: hit xyz, X, Y, Z, LX, gamma
    size_t cap;     // >= pixels of the launch
};
cudaError_t launch_hit(const VolumeDev& v, const ViewDev& view, HitRecords rec, float4* accum, cudaStream_t s);
// GatherData: 773 tile features per tile of a view.width x view.height grid.
cudaError_t launch_gather_tiles(const VolumeDev& v, const ViewDev& view, int px, int py, const float nl[3], float* out,
                                cudaStream_t s);
// fp16 = false: fp32 features (the FP32 network's input); true: fp16 pairs
// (the tensor-core networks' input, half the bytes), in the same buffer.
cudaError_t launch_gather_rec(const VolumeDev& v, const ViewDev& view, HitRecords rec, float* feat, bool fp16,
                              cudaStream_t s);
cudaError_t launch_mlp_rec_fp32(const VolumeDev& v, const ViewDev& view, HitRecords rec, const float* feat,
                                const float* weights, float4* accum, cudaStream_t s);
// Scatters records and tiled features to per-pixel layout (debug entry).
// feat in the gather's fp32 or fp16-pair layout (launch_gather_rec)
cudaError_t launch_debug_scatter(HitRecords rec, const float* feat, bool fp16, int npix, float* aux, float* feat_out,
                                 cudaStream_t s);
// Tiled feature buffer size for n records (floats).
inline size_t tiled_feature_floats(size_t n) { return ((n + 31) / 32) * 32 * 576; }

// gather_tex.cu: fp16 array copies of linear fp32 levels behind
// hardware-filtered textures (trilinear, normalized coordinates, border or
// clamp addressing) for the texture-unit gather, and of the HG LUT
// (bilinear, clamp).
struct GtexLevel {
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    cudaSurfaceObject_t surf = 0;   // the fill kernel's view of arr
    int n = 0;                      // edge: n^3 texels, or n x n for a flat level
    bool flat = false;
};
cudaError_t gtex_alloc_level(int n, bool clamp, GtexLevel* L);
cudaError_t gtex_alloc_lut(GtexLevel* L);
void gtex_free(GtexLevel* L);
// levels[i] <- src[i] (n^3 fp32, z fastest; a flat level 512 x 512, u
// fastest), rounded to fp16, in one launch per nine levels
cudaError_t gtex_fill(const GtexLevel* const* levels, const float* const* src, int count, int sms, cudaStream_t s);
size_t gtex_level_bytes(int n);
// The (mip L, TR L - 1) pair levels of the gather, L = 1..kGtexPairs-1
// (index 0 unused): half2 texels on an (n+2)^3 grid padded with the mip's
// border value and the TR level's clamp value, clamp addressing,
// unnormalized coordinates (texel centre of voxel i at i + 1.5).
cudaError_t gtex_alloc_pair(int n, GtexLevel* L);
cudaError_t gtex_fill_pairs(const GtexLevel* pairs, const float* mips, const float* trs, int sms, cudaStream_t s);
size_t gtex_pair_bytes(int n);

// tracer_kernels.cu: one launch of RenderCamera<false> (spp samples per
// pixel); FP64 sums of per-sample radiance and of its square per pixel.
// first_pos[pix] must start at spp and counter at 0.
cudaError_t launch_trace(const VolumeDev& v, const ViewDev& view, double* sum3, double* sumsq3, int* first_pos,
                         unsigned long long* counter, int sms, cudaStream_t s);
cudaError_t launch_fill_int(int* p, int n, int value, cudaStream_t s);
// GetSamples / GetTrs (core/volume.cu:710-834): one thread per task.
cudaError_t launch_get_samples(const VolumeDev& v, const float* alpha, const float* ori, const float* dir,
                               const float* ldir, const float* g, const float* scatter, int n, const float lc[3],
                               int multi_scatter, int spp, uint32_t seed, float* out3, cudaStream_t s);
cudaError_t launch_get_trs(const VolumeDev& v, float alpha, const float* ori, const float* dir, int n, const float L[3],
                           const float lc[3], float g, int spp, uint32_t seed, float* out3, cudaStream_t s);
cudaError_t launch_trace_resolve(const double* sum3, const int* first_pos, int npix, int spp, int frame, float4* accum,
                                 cudaStream_t s);

}  // namespace mrp
