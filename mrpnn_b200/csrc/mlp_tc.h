// mlp_tc.h -- tensor-core (tcgen05) forms of the MRPNN predictor MLP:
// BF16 and FP8-E4M3 operands with FP32 accumulation in TMEM.
#pragma once
#include "common.cuh"

namespace mrp {

// Weight images for the tensor-core kernels, built once per model.
struct TcWeights {
    void* d_bf16 = nullptr;    // BF16 operand images of the 58 tensor-core layers
    void* d_fp8 = nullptr;     // FP8-E4M3 operand images (weights / per-layer scale)
    float* d_scales = nullptr; // FP8 weight scales per output channel (row amax / 448)
    const float* d_fp32 = nullptr;   // packed fp32 weights: gates, biases, LSEFin, LX12
    float* d_aux = nullptr;    // fp32 constants of the CUDA-core parts, staged into shared memory
    int* d_err = nullptr;      // set to 1 when an MMA round times out
    int* d_counter = nullptr;  // tile counter of the persistent kernel
    bool ready = false;
};
// Per-handle scratch of the tensor-core predictor: the persistent kernel's
// tile counter (d[0]) and error flag (d[1]).  Every stream that launches the
// network needs its own, or two launches would share one tile counter.
struct TcScratch {
    int* d = nullptr;
};
// One request's staged records for the network: hit records, tiled features,
// running-mean image and the constants of its launch.  The batched launch
// takes up to kTcMaxSegments of them (each request's tiles stay separate).
struct TcSegment {
    const float* feat;           // the gather's FP16-pair tiled features (launch_gather_rec, fp16)
    const int* rec_count;
    const int* rec_pix;
    const float* rec_f;
    size_t rec_cap;
    float4* accum;
    f3 sr;                       // network input sigma = scatter_rate / 1.001
    f3 light_color, scatter_rate, ori;
    float g;
    int mean_k;
};
constexpr int kTcMaxSegments = 64;
struct HitRecords;
TcSegment tc_segment(const VolumeDev& v, const ViewDev& view, const HitRecords& rec, const float* feat,
                     float4* accum);
cudaError_t tc_prepare_weights(const float* packed_fp32_host, TcWeights& w);
cudaError_t tc_ensure_scratch(TcScratch& s);
void tc_free_scratch(TcScratch& s);
cudaError_t tc_launch_mlp(const TcWeights& w, bool fp8, const float* feat, const float* gamma, float g, const float sr[3],
                          int n, float* out3, int sms, cudaStream_t s);
// Same launch with the tile counter and the error flag at caller-given device
// addresses instead of the ones in TcWeights (both zeroed on `s` first).
cudaError_t tc_launch_mlp_at(const TcWeights& w, bool fp8, const float* feat, const float* gamma, float g,
                             const float sr[3], int n, float* out3, int* tile_counter, int* err, int sms,
                             cudaStream_t s);
// Network on the staged predictor's records and tiled features (kernels.h).
cudaError_t tc_launch_mlp_rec(const TcWeights& w, bool fp8, const VolumeDev& v, const ViewDev& view,
                              const HitRecords& rec, const float* feat, float4* accum, const TcScratch& sc, int sms,
                              cudaStream_t s);
// The network over several requests' records in one persistent launch:
// d_segs[0, nseg) in device memory (nseg <= kTcMaxSegments).
cudaError_t tc_launch_mlp_segments(const TcWeights& w, bool fp8, const TcSegment* d_segs, int nseg,
                                   const TcScratch& sc, int sms, cudaStream_t s);

// Self-test: D[128][n] = A[128][k] * B[n][k]^T with operands rounded to BF16
// (or E4M3), k a multiple of 16 (32), n a multiple of 16 up to 128.
cudaError_t tc_gemm_test(bool fp8, const float* A, const float* B, int n, int k, float* D, int* err, cudaStream_t s);

}  // namespace mrp
