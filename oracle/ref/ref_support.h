// ref_support.h -- shared pieces of the CPU checker build of the reference
// (oracle/_ref): the RNG stream selector and the warp emulation that the
// harnesses use.  TEST INFRASTRUCTURE ONLY.
#pragma once
#include <barrier>
#include <cstdint>
#include <thread>
#include <vector>

// Selects the Philox stream the next curand_init hands out (same definition
// as the oracle and the kernels: key = (id, seed ^ kind*0x9E3779B9),
// counter = (n/4, sub, frame, kind)).
void ref_set_stream(uint32_t kind, uint32_t id, uint32_t sub, uint32_t frame, uint32_t seed);

#if __cplusplus > 201703L
struct Warp {
    std::barrier<> bar{32};
    float f[2][32];
    unsigned u[2][32];
};
extern thread_local Warp* t_warp;
extern thread_local int t_lane, t_phase, t_shfl_slot;

// Run body(i, valid) for i in [0, n) as warps of 32 lanes (padding lanes run
// with valid=false and index 0 so that collectives stay complete).
template <class F>
inline void run_warps(int n, F body) {
    for (int base = 0; base < n; base += 32) {
        Warp w;
        std::vector<std::thread> lanes;
        for (int l = 0; l < 32; ++l) {
            lanes.emplace_back([&, l] {
                t_warp = &w; t_lane = l; t_phase = 0; t_shfl_slot = -1;
                int i = base + l;
                body(i < n ? i : base, i < n);
                t_warp = nullptr;
            });
        }
        for (auto& t : lanes) t.join();
    }
}
#endif
