// mlp_tc.cu -- tensor-core MLP (placeholder until the tcgen05 kernels land:
// every launch reports cudaErrorNotSupported, there is no fallback).
#include "mlp_tc.h"

namespace mrp {

cudaError_t tc_prepare_weights(const float*, TcWeights& w) { w.ready = false; return cudaSuccess; }
cudaError_t tc_ensure_scratch(TcScratch&, size_t) { return cudaSuccess; }
void tc_free_scratch(TcScratch& s) { if (s.buf) cudaFree(s.buf); s.buf = nullptr; s.bytes = 0; }
cudaError_t tc_launch_mlp(const TcWeights&, bool, const float*, const float*, float, const float*, int, float*, int,
                          cudaStream_t) {
    return cudaErrorNotSupported;
}
cudaError_t tc_launch_mlp_rec(const TcWeights&, bool, const VolumeDev&, const ViewDev&, const HitRecords&,
                              const float*, float4*, int, cudaStream_t) {
    return cudaErrorNotSupported;
}

}  // namespace mrp
