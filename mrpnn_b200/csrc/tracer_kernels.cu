// tracer_kernels.cu -- the delta-tracking path tracer (PT render mode), the
// ground-truth oracle of the renderer.
//
// Reference: RenderCamera<false> -> CalculateRadiance (core/volume.cu:198-228,
// core/render.cuh:535-597), free flights by DeterminateNextVertex
// (core/render.cuh:399-434) with NEE through the baked transmittance grid
// (nee_mode 0, the reference) or one unbiased Tr() estimate per vertex from
// the sample's own NEE stream (nee_mode 1; the error reference).
//
// B200 form: a persistent kernel pulls (pixel, sample) work items from a
// global counter, so a lane whose path ended starts the next one instead of
// idling until the longest path of its warp finishes (per-pixel threads
// leave most lanes idle: path lengths range from 0 to 256 bounces).  Every
// sample has its own Philox stream (sub = sample index), so results do not
// depend on which lane ran it.  Per-sample radiance is computed in fp32 in
// the reference's order and accumulated per pixel in FP64.
#include "kernels.h"
#include "tracing.cuh"

namespace mrp {


template <bool COUNT>
__global__ void __launch_bounds__(128, 8) k_trace(VolumeDev v, ViewDev w, double* __restrict__ sum3,
                                               double* __restrict__ sumsq3, int* __restrict__ first_pos,
                                               unsigned long long* __restrict__ counter) {
    const long long total = (long long)w.width * w.height * w.spp;
    const int npix = w.width * w.height;
    f3 L = normalize(w.light_dir);
    Tally tally;
    for (;;) {
        long long item;
        // one atomic per warp, items handed out in warp-sized runs
        unsigned lane = threadIdx.x & 31;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        item = (long long)base + lane;
        if ((long long)base >= total) break;
        if (item >= total) continue;
        // sample-major order: consecutive lanes trace neighbouring pixels
        int k = (int)(item / npix), pix = (int)(item % npix);
        int row = pix / w.width, col = pix % w.width;
        f3 ori = w.ori, dir;
        if (w.ray_dir) {   // GetRadiances: explicit rays
            ori = mk3(w.ray_ori[3 * pix], w.ray_ori[3 * pix + 1], w.ray_ori[3 * pix + 2]);
            dir = normalize(mk3(w.ray_dir[3 * pix], w.ray_dir[3 * pix + 1], w.ray_dir[3 * pix + 2]));
        } else {
            dir = normalize(camera_ray_t(w, row, col));
        }
        float dis = ray_box_offset(ori, dir);
        f3 r;
        if (dis < 0) {
            r = v.sky;   // SkyBox(dir), coverage stays 0
        } else {
            r = trace_sample(v, w, pix, k, ori, dir, dis, L, COUNT ? &tally : nullptr);
            if (COUNT) tally.events++;
            if (r.x > 0 || r.y > 0 || r.z > 0) atomicMin(first_pos + pix, k);
        }
        atomicAdd(sum3 + 3 * pix, (double)r.x);
        atomicAdd(sum3 + 3 * pix + 1, (double)r.y);
        atomicAdd(sum3 + 3 * pix + 2, (double)r.z);
        if (sumsq3) {
            atomicAdd(sumsq3 + 3 * pix, (double)r.x * r.x);
            atomicAdd(sumsq3 + 3 * pix + 1, (double)r.y * r.y);
            atomicAdd(sumsq3 + 3 * pix + 2, (double)r.z * r.z);
        }
    }
    if (COUNT) flush_tally(w.counters, tally);
}

// GetSample (core/render.cuh:615-655), the training-data generator: one
// thread per task; the first direction HG-sampled around dir, up to
// multi_scatter bounces, NEE by Tr() on the task's one stream (kind 4).
struct SampleTasks {
    const float *alpha, *ori, *dir, *ldir, *g, *scatter;
    int n;
    f3 light_color;
    int multi_scatter, spp;
    uint32_t seed;
};
__global__ void __launch_bounds__(128) k_get_samples(VolumeDev v, SampleTasks T, float* __restrict__ out3) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= T.n) return;
    Stream st(kSampleStream, (uint32_t)q, 0, 0, T.seed);
    f3 o = mk3(T.ori[3 * q], T.ori[3 * q + 1], T.ori[3 * q + 2]);
    f3 d = mk3(T.dir[3 * q], T.dir[3 * q + 1], T.dir[3 * q + 2]);
    f3 L = mk3(T.ldir[3 * q], T.ldir[3 * q + 1], T.ldir[3 * q + 2]);
    float a = T.alpha[q], gq = T.g[q], sc = T.scatter[q];
    f3 res = mk3(0, 0, 0);
    for (int i = 0; i < T.spp; ++i) {
        f3 pos = o;
        float e1 = st.next();
        float e0 = st.next();
        f3 rd = sample_hg(e0, e1, d, gq);
        f3 csr = mk3(1, 1, 1);
        for (int b = 0; b < T.multi_scatter; ++b) {
            f3 np, nd;
            float dis = ray_box_distance(pos, rd);
            if (!next_vertex(v, st, a, gq, pos, rd, dis, &np, &nd, nullptr)) {
                res = add(res, mul(v.sky, csr));
                break;
            }
            pos = np;
            csr = mul(mul(csr, 1.001f), sc);
            dis = ray_box_distance(pos, L);
            float phase = hg(dot(rd, L), gq);
            res = add(res, mul(mul(T.light_color, csr), fm(transmittance(v, st, pos, L, dis, a), phase)));
            rd = nd;
        }
    }
    float fs_ = (float)T.spp;
    out3[3 * q] = fd(res.x, fs_);
    out3[3 * q + 1] = fd(res.y, fs_);
    out3[3 * q + 2] = fd(res.z, fs_);
}

// GetTrs -> ShadowTerm_TRs (core/render.cuh:668-680): light colour x pi x the
// mean of Tr() x HG over spp estimates from the task's stream (kind 5).
__global__ void __launch_bounds__(128) k_get_trs(VolumeDev v, float alpha, const float* __restrict__ ori,
                                                 const float* __restrict__ dir, int n, f3 L, f3 lc, float g, int spp,
                                                 uint32_t seed, float* __restrict__ out3) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    Stream st(kTrStream, (uint32_t)q, 0, 0, seed);
    f3 o = mk3(ori[3 * q], ori[3 * q + 1], ori[3 * q + 2]);
    f3 d = mk3(dir[3 * q], dir[3 * q + 1], dir[3 * q + 2]);
    float res = 0.0f;
    for (int i = 0; i < spp; ++i) {
        float dis = ray_box_distance(o, L);
        float phase = hg(dot(d, L), g);
        res = fa(res, fm(transmittance(v, st, o, L, dis, alpha), phase));
    }
    f3 r = mul(lc, 3.1415926535f);
    float fs_ = (float)spp;
    out3[3 * q] = fd(fm(r.x, res), fs_);
    out3[3 * q + 1] = fd(fm(r.y, res), fs_);
    out3[3 * q + 2] = fd(fm(r.z, res), fs_);
}

// (mean radiance, coverage) of the launch, then the running mean over
// launches (core/volume.cu:224-227).  Coverage: the reference counts samples
// after which its running radiance sum is positive (core/render.cuh:594).
__global__ void k_trace_resolve(const double* __restrict__ sum3, const int* __restrict__ first_pos, int npix, int spp,
                                int frame, float4* __restrict__ accum) {
    int pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= npix) return;
    float4 res;
    res.x = (float)(sum3[3 * pix] / spp);
    res.y = (float)(sum3[3 * pix + 1] / spp);
    res.z = (float)(sum3[3 * pix + 2] / spp);
    int kf = first_pos[pix];
    res.w = kf < spp ? fd((float)(spp - kf), (float)spp) : 0.0f;
    res.x = fmaxf(0.0f, res.x); res.y = fmaxf(0.0f, res.y); res.z = fmaxf(0.0f, res.z);
    float rate = fd(1.0f, (float)(1 + frame));
    float4 a = frame == 0 ? make_float4(0, 0, 0, 0) : accum[pix];
    accum[pix] = make_float4(lerp(a.x, res.x, rate), lerp(a.y, res.y, rate), lerp(a.z, res.z, rate), lerp(a.w, res.w, rate));
}

__global__ void k_fill_int(int* __restrict__ p, int n, int value) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = value;
}
cudaError_t launch_fill_int(int* p, int n, int value, cudaStream_t s) {
    if (n > 0) k_fill_int<<<(n + 255) / 256, 256, 0, s>>>(p, n, value);
    return cudaGetLastError();
}

cudaError_t launch_trace(const VolumeDev& v, const ViewDev& view, double* sum3, double* sumsq3, int* first_pos,
                         unsigned long long* counter, int sms, cudaStream_t s) {
    if (view.counters) k_trace<true><<<sms * 8, 128, 0, s>>>(v, view, sum3, sumsq3, first_pos, counter);
    else k_trace<false><<<sms * 8, 128, 0, s>>>(v, view, sum3, sumsq3, first_pos, counter);
    return cudaGetLastError();
}
cudaError_t launch_get_samples(const VolumeDev& v, const float* alpha, const float* ori, const float* dir,
                               const float* ldir, const float* g, const float* scatter, int n, const float lc[3],
                               int multi_scatter, int spp, uint32_t seed, float* out3, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    SampleTasks T{alpha, ori, dir, ldir, g, scatter, n, mk3(lc[0], lc[1], lc[2]), multi_scatter, spp, seed};
    k_get_samples<<<(n + 127) / 128, 128, 0, s>>>(v, T, out3);
    return cudaGetLastError();
}
cudaError_t launch_get_trs(const VolumeDev& v, float alpha, const float* ori, const float* dir, int n, const float L[3],
                           const float lc[3], float g, int spp, uint32_t seed, float* out3, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_get_trs<<<(n + 127) / 128, 128, 0, s>>>(v, alpha, ori, dir, n, mk3(L[0], L[1], L[2]), mk3(lc[0], lc[1], lc[2]),
                                               g, spp, seed, out3);
    return cudaGetLastError();
}
cudaError_t launch_trace_resolve(const double* sum3, const int* first_pos, int npix, int spp, int frame, float4* accum,
                                 cudaStream_t s) {
    k_trace_resolve<<<(npix + 255) / 256, 256, 0, s>>>(sum3, first_pos, npix, spp, frame, accum);
    return cudaGetLastError();
}

}  // namespace mrp
