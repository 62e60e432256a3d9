// tracer_kernels.cu -- the delta-tracking path tracer (PT render mode), the
// ground-truth oracle of the renderer.
//
// Reference: RenderCamera<false> -> CalculateRadiance (core/volume.cu:198-228,
// core/render.cuh:535-597), free flights by DeterminateNextVertex
// (core/render.cuh:399-434) with NEE through the baked transmittance grid
// (nee_mode 0, the reference) or one unbiased Tr() estimate per vertex from
// the sample's own NEE stream (nee_mode 1; the error reference).
//
// B200 form: a persistent kernel runs an event loop per lane.  A lane holds
// one (pixel, sample) item; one loop iteration of a warp is either a
// free-flight step (two draws, one density fetch, one comparison) of every
// lane that is in flight, or the real-collision work (phase sampling, NEE,
// next flight) of every lane that has collided.  Collided lanes wait until
// kScatterBatch of them are pending (or no lane can step), so the long
// collision branch runs with many lanes at once instead of with the one or
// two that collide in a given step.  A lane whose sample ends takes the next
// item from a global counter at once (one atomic per warp for all lanes
// that need work).  Every sample has its own Philox stream (sub = sample
// index) and its arithmetic is CalculateRadiance's, in the reference's order,
// so results do not depend on which lane ran it or when.  The free-flight
// step (distance and accept test) uses the fast log and division that the
// reference's -use_fast_math build compiles to (CMakeLists.txt:184); the
// rest is in IEEE float.  Per-sample radiance is fp32, accumulated per pixel
// in FP64.
#include "kernels.h"
#include "tracing.cuh"

namespace mrp {

namespace {
constexpr int kScatterBatch = 8;

// The sample's kPixelStream: the state of Stream(kPixelStream, pix, k,
// frame, seed) without its constant fields (same draws).
struct LaneStream {
    uint32_t n, blk[4];
    MRP_D float next(uint32_t pix, uint32_t k, uint32_t frame, uint32_t seed) {
        if ((n & 3) == 0) philox(n >> 2, k, frame, kPixelStream, pix, seed ^ (kPixelStream * 0x9E3779B9u), blk);
        uint32_t x = (n & 2) ? ((n & 1) ? blk[3] : blk[2]) : ((n & 1) ? blk[1] : blk[0]);
        ++n;
        return u01(x);
    }
};

// nee_mode 1: one unbiased Tr() estimate from the sample's NEE stream,
// positioned at draw *n.
template <class DT>
__device__ __forceinline__ float nee_tr(const VolumeDev& v, const ViewDev& w, int pix, int k, uint32_t* n, f3 p, f3 L) {
    Stream s(kNeeStream, (uint32_t)pix, (uint32_t)k, (uint32_t)w.frame, w.seed);
    s.n = *n;
    if (s.n & 3) philox(s.n >> 2, s.sub, s.frame, s.kind, s.k0, s.k1, s.blk);
    float tr = transmittance<DT>(v, s, p, L, ray_box_distance(p, L), w.alpha);
    *n = s.n;
    return tr;
}

MRP_D void deposit(double* __restrict__ sum3, double* __restrict__ sumsq3, int* __restrict__ first_pos, int pix, int k,
                   f3 r, bool hit) {
    if (hit && (r.x > 0 || r.y > 0 || r.z > 0)) atomicMin(first_pos + pix, k);
    atomicAdd(sum3 + 3 * pix, (double)r.x);
    atomicAdd(sum3 + 3 * pix + 1, (double)r.y);
    atomicAdd(sum3 + 3 * pix + 2, (double)r.z);
    if (sumsq3) {
        atomicAdd(sumsq3 + 3 * pix, (double)r.x * r.x);
        atomicAdd(sumsq3 + 3 * pix + 1, (double)r.y * r.y);
        atomicAdd(sumsq3 + 3 * pix + 2, (double)r.z * r.z);
    }
}
}  // namespace

template <bool COUNT, class DT, bool TEX = false, bool ENV = false>
__global__ void __launch_bounds__(128, 8) k_trace(const __grid_constant__ VolumeDev v,
                                               const __grid_constant__ ViewDev w, double* __restrict__ sum3,
                                               double* __restrict__ sumsq3, int* __restrict__ first_pos,
                                               unsigned long long* __restrict__ counter) {
    const unsigned long long total = (unsigned long long)w.width * w.height * w.spp;
    const int npix = w.width * w.height;
    const f3 L = normalize(w.light_dir);
    const float smax = fm(v.max_density, w.alpha);
    const uint32_t frame = (uint32_t)w.frame, seed = w.seed;
    const unsigned lane = threadIdx.x & 31, lt_mask = (1u << lane) - 1u;
    Tally tally;
    // the lane's sample: pixel, index, stream, vertex, direction, throughput,
    // radiance, bounce, free-flight distance / limit / iteration
    bool live = false, dry = false, hit = false;
    int pix = 0, k = 0, b = 0, loop = 0;
    uint32_t nee_n = 0;
    LaneStream st{0, {0, 0, 0, 0}};
    f3 p = mk3(0, 0, 0), rd = p, csr = p, res = p;
    float t = 0.0f, md = 0.0f;
    for (;;) {
        // refill: every lane without a sample takes the next item (rays that
        // miss the box are resolved to the sky here and refilled again)
        for (;;) {
            const unsigned need = __ballot_sync(0xffffffffu, !live && !dry);
            if (!need) break;
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!live && !dry) {
                const unsigned long long item = base + __popc(need & lt_mask);
                if (item >= total) {
                    dry = true;
                } else {
                    // sample-major order: consecutive items trace neighbouring pixels
                    k = (int)(item / npix);
                    pix = (int)(item % npix);
                    int row = pix / w.width, col = pix % w.width;
                    f3 ori = w.ori, dir;
                    if (w.ray_dir) {   // GetRadiances: explicit rays
                        ori = mk3(w.ray_ori[3 * pix], w.ray_ori[3 * pix + 1], w.ray_ori[3 * pix + 2]);
                        dir = normalize(mk3(w.ray_dir[3 * pix], w.ray_dir[3 * pix + 1], w.ray_dir[3 * pix + 2]));
                    } else {
                        dir = normalize(camera_ray_t(w, row, col));
                    }
                    float dis = ray_box_offset(ori, dir);
                    if (dis < 0) {
                        deposit(sum3, sumsq3, first_pos, pix, k, ENV ? sky_map(v.hdri, v.hdri_w, v.hdri_h, v.env_exp, dir) : v.sky,
                                false);   // SkyBox(dir), coverage stays 0
                    } else {
                        if (COUNT) tally.events++;
                        if (w.multi_scatter < 1) {
                            deposit(sum3, sumsq3, first_pos, pix, k, mk3(0, 0, 0), true);
                        } else {
                            st.n = 0;
                            nee_n = 0;
                            res = mk3(0, 0, 0);
                            p = add(ori, mul(dir, dis));
                            rd = dir;
                            csr = mk3(1, 1, 1);
                            b = 0;
                            md = ray_box_distance(p, rd);
                            t = 0.0f;
                            loop = 0;
                            hit = false;
                            if (COUNT) tally.steps++;
                            live = true;
                        }
                    }
                }
            }
        }
        const unsigned pend = __ballot_sync(0xffffffffu, live && hit);
        const unsigned fly = __ballot_sync(0xffffffffu, live && !hit);
        if (!(pend | fly)) break;
        if (fly && __popc(pend) < kScatterBatch) {
            if (!live || hit) continue;
            // one iteration of DeterminateNextVertex's loop (while (loop++ < 10000))
            if (loop >= 10000) { hit = true; continue; }
            ++loop;
            float rk = st.next(pix, k, frame, seed);
            // the free-flight step in the reference's build arithmetic
            // (-use_fast_math: __logf, __fdividef), 10 % of the frame
            // against IEEE log and division; decisions stay per sample
            t = t - __fdividef(__logf(1.0f - rk), smax);
            if (t > md) {   // left the box: sky radiance, the sample ends
                res = add(res, mul(ENV ? sky_map(v.hdri, v.hdri_w, v.hdri_h, v.env_exp, rd) : v.sky, csr));
                deposit(sum3, sumsq3, first_pos, pix, k, res, true);
                live = false;
                continue;
            }
            rk = st.next(pix, k, frame, seed);
            const f3 q = add(p, mul(rd, t));
            // the texture unit's filter (tracer_filter 1), as the reference's
            // Density(): tex3D(uv.z, uv.y, uv.x) with uv = pos + 0.5
            float d = TEX ? tex3D<float>(v.dens_tex, q.z + 0.5f, q.y + 0.5f, q.x + 0.5f) : density_t<DT>(v, q);
            if (COUNT) tally.fetches++;
            float S = d * w.alpha;
            hit = __fdividef(S, smax) > rk;
            if (!hit && d < 0) t = fs(t, d);
            continue;
        }
        if (!live || !hit) continue;
        // real collision: phase sampling, NEE, next flight
        float e1 = st.next(pix, k, frame, seed);
        float e0 = st.next(pix, k, frame, seed);
        f3 nd = sample_hg(e0, e1, rd, w.g);
        p = add(mul(rd, t), p);
        csr = mul(csr, v.scatter_rate);
        float ph = hg(dot(rd, L), w.g);
        // NEE: MipTr(0, p) on the baked grid (core/render.cuh:589), through
        // the texture unit under tracer_filter as the reference's tex3D
        float tr = v.nee_mode ? nee_tr<DT>(v, w, pix, k, &nee_n, p, L)
                 : TEX && v.baked_tex ? tex3D<float>(v.baked_tex, p.z + 0.5f, p.y + 0.5f, p.x + 0.5f)
                                      : tex3<true>(v.baked, v.baked_res, p);
        if (COUNT) tally.lookups++;
        res = add(res, mul(mul(w.light_color, csr), fm(tr, ph)));
        rd = nd;
        hit = false;
        if (++b >= w.multi_scatter) {
            deposit(sum3, sumsq3, first_pos, pix, k, res, true);
            live = false;
        } else {
            md = ray_box_distance(p, rd);
            t = 0.0f;
            loop = 0;
            if (COUNT) tally.steps++;
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
                res = add(res, mul(sky_radiance(v, rd), csr));
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

// One copy of the event loop per density storage type and: counting mode,
// the free flight through the density texture (tracer_filter), an
// environment map (its lookup is a call, which costs the loop registers
// where it is compiled in).  The counting copy ignores the map: the work it
// counts does not depend on the sky, and its image is not kept.
template <class DT>
static void launch_trace_dt(const VolumeDev& v, const ViewDev& view, double* sum3, double* sumsq3, int* first_pos,
                            unsigned long long* counter, int sms, cudaStream_t s) {
    const dim3 grid(sms * 8), block(128);
    if (view.counters) k_trace<true, DT><<<grid, block, 0, s>>>(v, view, sum3, sumsq3, first_pos, counter);
    else if (v.dens_tex && v.hdri) k_trace<false, DT, true, true><<<grid, block, 0, s>>>(v, view, sum3, sumsq3, first_pos, counter);
    else if (v.dens_tex) k_trace<false, DT, true, false><<<grid, block, 0, s>>>(v, view, sum3, sumsq3, first_pos, counter);
    else if (v.hdri) k_trace<false, DT, false, true><<<grid, block, 0, s>>>(v, view, sum3, sumsq3, first_pos, counter);
    else k_trace<false, DT><<<grid, block, 0, s>>>(v, view, sum3, sumsq3, first_pos, counter);
}
cudaError_t launch_trace(const VolumeDev& v, const ViewDev& view, double* sum3, double* sumsq3, int* first_pos,
                         unsigned long long* counter, int sms, cudaStream_t s) {
    if (v.density_h) launch_trace_dt<__half>(v, view, sum3, sumsq3, first_pos, counter, sms, s);
    else launch_trace_dt<float>(v, view, sum3, sumsq3, first_pos, counter, sms, s);
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
