// mlp_tc.h -- tensor-core (tcgen05) forms of the MRPNN predictor MLP:
// BF16 and FP8-E4M3 operands with FP32 accumulation in TMEM.
#pragma once
#include "common.cuh"

namespace mrp {

// Weight images for the tensor-core kernels, built once per model.
struct TcWeights {
    void* d_bf16 = nullptr;    // packed BF16 operand tiles
    void* d_fp8 = nullptr;     // packed FP8 operand tiles
    float* d_scales = nullptr; // per-layer FP8 dequantisation scales
    float* d_fp32 = nullptr;   // fp32 weights for the CUDA-core parts (gates)
    bool ready = false;
};
// Per-handle scratch of the tensor-core predictor.
struct TcScratch {
    void* buf = nullptr;
    size_t bytes = 0;
};

cudaError_t tc_prepare_weights(const float* packed_fp32_host, TcWeights& w);
cudaError_t tc_ensure_scratch(TcScratch& s, size_t npix);
void tc_free_scratch(TcScratch& s);
cudaError_t tc_launch_mlp(const TcWeights& w, bool fp8, const float* feat, const float* gamma, float g, const float sr[3],
                          int n, float* out3, int sms, cudaStream_t s);
// Network on the staged predictor's records and tiled features (kernels.h).
struct HitRecords;
cudaError_t tc_launch_mlp_rec(const TcWeights& w, bool fp8, const VolumeDev& v, const ViewDev& view,
                              const HitRecords& rec, const float* feat, float4* accum, int sms, cudaStream_t s);

}  // namespace mrp
