// serve.cu -- the serving loop of include/mrpnn.h (mrp_serve_*): resident
// volumes, MRPNN render requests admitted into device slots by a memory
// budget, per-request first hit + gather on the slot's stream, and the
// network of every request whose features are ready in one batched
// persistent tcgen05 launch (continuous batching).
//
// The reference has no counterpart: VolumeRender::Render renders one frame
// per synchronous call (core/volume.cu:487-548).  Each result here is the
// one mrp_render gives for the same view with sample_num 1: the same
// kernels on the same per-pixel streams; only the network launch is shared.
//
// Threads.  API calls only touch the ticket table under `mu`; one worker
// thread owns every CUDA call of the server.  The worker polls events
// (cudaEventQuery) and sleeps 20 us when nothing moved, so no wait of the
// server can hang: the GPU work it waits for is ordinary bounded kernels.
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "abi_internal.h"

using namespace mrpi;

namespace {
using Clock = std::chrono::steady_clock;

struct Ticket {
    uint64_t id = 0;
    mrp_request req{};
    size_t npix = 0;
    bool done = false;
    mrp_status status = MRP_OK;
    std::string error;
    mrp_request_timing t{};
};

enum SlotState { kFree, kFeatures, kNetwork, kOutput };

// Device working set of one admitted request.  Buffers grow to the largest
// request the slot has held and are kept; the budget counts what is held.
struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_feat = nullptr, ev_done = nullptr;
    size_t cap = 0, bytes = 0;
    float* trs = nullptr;          // this request's TR mips (kTrFloats)
    int* rec_count = nullptr;
    int* rec_pix = nullptr;
    float* rec_f = nullptr;
    float* feat = nullptr;
    float4* accum = nullptr;
    GtexLevel gtr0;                // texture copies of TR level 0 and of the (mip, TR) pairs of this
    GtexLevel gpair[kGtexPairs];   // request (tensor-core servers; gtr0.arr null until used)
    float* staging = nullptr;      // pinned host copy for pageable outputs
    size_t staging_cap = 0;
    bool staged_out = false;
    SlotState state = kFree;
    std::shared_ptr<Ticket> t;
    VolumeDev vd{};
    ViewDev view{};
    HitRecords records() const { return HitRecords{rec_count, rec_pix, rec_f, cap}; }
};

size_t slot_bytes(size_t npix) {
    return kTrFloats * sizeof(float) + 2 * sizeof(int) + npix * (sizeof(int) + 16 * sizeof(float) + sizeof(float4)) +
           tiled_feature_floats(npix) * sizeof(float);
}
constexpr size_t kLutBytes = kLutAlloc * sizeof(float);   // the LUT and its lut_dirs table

struct Lut {
    float g;
    uint32_t seed;
    float* d;
    cudaEvent_t ready;
    GtexLevel tex;   // its texture copy (tensor-core servers)
};

// Texture copy of one volume's mip level 0 for the texture-unit gather,
// shared by every request on that volume; rebuilt when the volume's pyramid
// is (version), given back under budget pressure when no slot uses them.
struct VolTex {
    uint64_t uid = 0;
    unsigned version = 0;
    GtexLevel mip0;
    cudaEvent_t ready = nullptr;
    int users = 0;
};
size_t tr_tex_bytes() {   // a slot's: TR level 0 and the pairs
    size_t b = gtex_level_bytes(128);
    for (int l = 1; l < kGtexPairs; ++l) b += gtex_pair_bytes(256 >> l);
    return b;
}
size_t mip_tex_bytes() { return gtex_level_bytes(256); }
const size_t kLutTexBytes = (size_t)kLut * kLut * 2;

double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}
std::string cuda_msg(const char* what, cudaError_t e) { return std::string(what) + ": " + cudaGetErrorString(e); }
}  // namespace

struct mrp_server {
    mrp_serve_config cfg{};
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Ticket>> incoming;                    // guarded by mu
    std::unordered_map<uint64_t, std::shared_ptr<Ticket>> tickets;   // guarded by mu
    uint64_t next_id = 1;
    bool stopping = false;                                           // guarded by mu
    mrp_serve_stats stats{};                                         // guarded by mu
    Clock::time_point t0;
    // worker-only state
    std::deque<std::shared_ptr<Ticket>> pending;
    std::vector<Slot> slots;
    std::vector<Lut> luts;
    std::vector<std::unique_ptr<VolTex>> vtex;
    std::vector<VolTex*> slot_vtex;   // per slot: the pyramid textures its request holds, or null
    bool tex_mode = false;            // tensor-core network: the gather may sample textures
    size_t used = 0;
    cudaStream_t net = nullptr;
    cudaEvent_t ev_net = nullptr;
    TcScratch sc;
    TcSegment* d_segs = nullptr;
    TcSegment* h_segs = nullptr;   // pinned
    int* h_err = nullptr;          // pinned
    std::vector<int> batch;        // slots in the network launch in flight
    bool net_busy = false;

    void complete(const std::shared_ptr<Ticket>& T, mrp_status st, const std::string& err) {
        std::lock_guard<std::mutex> lk(mu);
        T->status = st;
        T->error = err;
        T->done = true;
        T->t.done_ms = ms_since(t0);
        if (st == MRP_OK) stats.completed++;
        else stats.failed++;
        stats.bytes_in_use = used;
        cv_done.notify_all();
    }
    void release(Slot& s) {
        VolTex*& vt = slot_vtex[&s - slots.data()];
        if (vt) vt->users--;
        vt = nullptr;
        s.state = kFree;
        s.t.reset();
        s.staged_out = false;
    }
    // Slot buffers are stream-ordered allocations on the slot's stream: a
    // slot that grows frees and allocates in stream order, without the
    // device-wide synchronisation of cudaFree.
    void free_buffers(Slot& s) {
        for (void* p : {(void*)s.trs, (void*)s.rec_count, (void*)s.rec_pix, (void*)s.rec_f, (void*)s.feat,
                        (void*)s.accum})
            if (p) mrp::dev_free_async(p, s.stream);
        s.trs = nullptr; s.rec_count = nullptr; s.rec_pix = nullptr; s.rec_f = nullptr; s.feat = nullptr;
        s.accum = nullptr;
        used -= s.bytes;
        s.bytes = 0;
        s.cap = 0;
        if (s.gtr0.arr) {   // arrays are not stream-ordered: the slot's work ends first
            cudaStreamSynchronize(s.stream);
            gtex_free(&s.gtr0);
            for (GtexLevel& L : s.gpair) gtex_free(&L);
            used -= tr_tex_bytes();
        }
    }
    cudaError_t ensure_tr_textures(Slot& s) {
        if (s.gtr0.arr) return cudaSuccess;
        cudaError_t e = gtex_alloc_level(128, true, &s.gtr0);
        for (int l = 1; l < kGtexPairs && e == cudaSuccess; ++l) e = gtex_alloc_pair(256 >> l, &s.gpair[l]);
        if (e != cudaSuccess) {
            gtex_free(&s.gtr0);
            for (GtexLevel& L : s.gpair) gtex_free(&L);
            return e;
        }
        used += tr_tex_bytes();
        return cudaSuccess;
    }
    VolTex* find_vtex(const mrp_volume* v) {
        for (auto& p : vtex)
            if (p->uid == v->uid) return p.get();
        return nullptr;
    }
    void drop_vtex(size_t i) {
        VolTex* p = vtex[i].get();
        if (p->ready) cudaEventSynchronize(p->ready);
        gtex_free(&p->mip0);
        if (p->ready) cudaEventDestroy(p->ready);
        used -= mip_tex_bytes();
        vtex.erase(vtex.begin() + (long)i);
    }
    VolTex* vtex_for(const mrp_volume* v, cudaStream_t st, std::string* err);
    cudaError_t grow(Slot& s, size_t npix) {
        free_buffers(s);
        cudaError_t e;
        if ((e = mrp::dev_malloc_async(&s.trs, kTrFloats * sizeof(float), s.stream)) != cudaSuccess ||
            (e = mrp::dev_malloc_async(&s.rec_count, 2 * sizeof(int), s.stream)) != cudaSuccess ||
            (e = mrp::dev_malloc_async(&s.rec_pix, npix * sizeof(int), s.stream)) != cudaSuccess ||
            (e = mrp::dev_malloc_async(&s.rec_f, npix * 16 * sizeof(float), s.stream)) != cudaSuccess ||
            (e = mrp::dev_malloc_async(&s.feat, tiled_feature_floats(npix) * sizeof(float), s.stream)) != cudaSuccess ||
            (e = mrp::dev_malloc_async(&s.accum, npix * sizeof(float4), s.stream)) != cudaSuccess) {
            free_buffers(s);
            return e;
        }
        s.cap = npix;
        s.bytes = slot_bytes(npix);
        used += s.bytes;
        return cudaSuccess;
    }

    bool admit();
    bool launch_network();
    bool finish_network();
    bool finish_outputs();
    void enqueue_output(Slot& s, bool after_net);
    const Lut* lut_for(float g_, uint32_t seed, cudaStream_t s, std::string* err);
    void run();
};

// The LUT of (g, seed), shared by every request that asks for it; built once
// on the stream of the first such request, which the others then wait for.
const Lut* mrp_server::lut_for(float g_, uint32_t seed, cudaStream_t s, std::string* err) {
    for (const Lut& l : luts)
        if (l.g == g_ && l.seed == seed) {
            cudaStreamWaitEvent(s, l.ready, 0);
            return &l;
        }
    Lut l{g_, seed, nullptr, nullptr, GtexLevel{}};
    cudaError_t e;
    if ((e = mrp::dev_malloc(&l.d, kLutBytes)) != cudaSuccess) { *err = cuda_msg("LUT", e); return nullptr; }
    const GtexLevel* lv = &l.tex;
    const float* src = l.d;
    if ((e = cudaEventCreateWithFlags(&l.ready, cudaEventDisableTiming)) != cudaSuccess ||
        (e = launch_hg_lut(l.d, g_, seed, s)) != cudaSuccess ||
        (e = launch_lut_dirs(l.d, l.d + kLut * kLut, s)) != cudaSuccess ||
        (tex_mode && ((e = gtex_alloc_lut(&l.tex)) != cudaSuccess || (e = gtex_fill(&lv, &src, 1, g.sms, s)) != cudaSuccess)) ||
        (e = cudaEventRecord(l.ready, s)) != cudaSuccess) {
        if (l.tex.arr) {
            cudaStreamSynchronize(s);
            gtex_free(&l.tex);
        }
        mrp::dev_free(l.d);
        if (l.ready) cudaEventDestroy(l.ready);
        *err = cuda_msg("LUT", e);
        return nullptr;
    }
    used += kLutBytes + (tex_mode ? kLutTexBytes : 0);
    luts.push_back(l);
    return &luts.back();
}

// The pyramid textures of volume v, built on the stream of the first request
// that asks for them (or after the volume's pyramid changed), which later
// requests wait for.  The caller counts the request as a user.
VolTex* mrp_server::vtex_for(const mrp_volume* v, cudaStream_t st, std::string* err) {
    VolTex* p = find_vtex(v);
    if (p && p->version == v->pyramid_version) {
        cudaStreamWaitEvent(st, p->ready, 0);
        return p;
    }
    cudaError_t e = cudaSuccess;
    if (!p) {
        auto q = std::make_unique<VolTex>();
        q->uid = v->uid;
        e = gtex_alloc_level(256, false, &q->mip0);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&q->ready, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            gtex_free(&q->mip0);
            *err = cuda_msg("pyramid textures", e);
            return nullptr;
        }
        used += mip_tex_bytes();
        vtex.push_back(std::move(q));
        p = vtex.back().get();
    } else {
        cudaStreamWaitEvent(st, p->ready, 0);   // a previous fill of the old pyramid
    }
    const GtexLevel* lv = &p->mip0;
    const float* src = v->mips;
    if ((e = gtex_fill(&lv, &src, 1, g.sms, st)) != cudaSuccess || (e = cudaEventRecord(p->ready, st)) != cudaSuccess) {
        *err = cuda_msg("pyramid textures", e);
        return nullptr;
    }
    p->version = v->pyramid_version;
    return p;
}

// Admission, first come first served: the head request enters when a slot
// is free and its working set fits the budget (idle slots give their buffers
// back first if needed).  Then its TR mips, first hit and gather are queued
// on the slot's stream.
bool mrp_server::admit() {
    bool moved = false;
    while (!pending.empty()) {
        std::shared_ptr<Ticket> T = pending.front();
        // a free slot whose buffers already hold the request (the smallest
        // such), else the free slot with the largest buffers (least growth)
        int pick = -1;
        for (int i = 0; i < (int)slots.size(); ++i) {
            const Slot& c = slots[i];
            if (c.state != kFree) continue;
            if (pick < 0) { pick = i; continue; }
            const Slot& b = slots[pick];
            bool c_fits = c.cap >= T->npix, b_fits = b.cap >= T->npix;
            if (c_fits != b_fits ? c_fits : (c_fits ? c.cap < b.cap : c.cap > b.cap)) pick = i;
        }
        if (pick < 0) break;
        Slot& s = slots[pick];
        mrp_volume* v = T->req.volume;
        // with an environment map the request's light is the map's or the
        // sun's, picked as mrp_render picks it for its launch
        mrp_view w = T->req.view;
        if (v->hdri) env_light_for_launch(v, (uint32_t)w.frame_offset, w.seed, w.light_dir, w.light_color);
        bool need_lut = true;
        for (const Lut& l : luts)
            if (l.g == w.g && l.seed == v->params.seed) need_lut = false;
        // the texture-unit gather (the volume's gather_filter) adds the
        // slot's TR textures, the volume's pyramid textures and the LUT's
        const bool use_tex = tex_mode && v->params.gather_filter;
        size_t need = (s.cap >= T->npix ? 0 : slot_bytes(T->npix) - s.bytes) +
                      (need_lut ? kLutBytes + (tex_mode ? kLutTexBytes : 0) : 0) +
                      (use_tex && !s.gtr0.arr ? tr_tex_bytes() : 0) + (use_tex && !find_vtex(v) ? mip_tex_bytes() : 0);
        if (used + need > cfg.memory_budget) {
            for (Slot& o : slots)   // idle slots give their buffers back
                if (&o != &s && o.state == kFree && (o.bytes || o.gtr0.arr) && used + need > cfg.memory_budget)
                    free_buffers(o);
            for (size_t i = vtex.size(); i-- > 0 && used + need > cfg.memory_budget;)   // and unused pyramid textures
                if (vtex[i]->users == 0 && vtex[i]->uid != v->uid) drop_vtex(i);
            bool busy = false;
            for (const Slot& o : slots) busy = busy || o.state != kFree;
            if (used + need > cfg.memory_budget && !busy) {   // nothing left to wait for
                pending.pop_front();
                moved = true;
                complete(T, MRP_ERR_BUDGET, "request does not fit the budget beside the server's caches");
                continue;
            }
            if (used + need > cfg.memory_budget) break;   // wait for running requests to finish
        }
        pending.pop_front();
        moved = true;
        T->t.admit_ms = ms_since(t0);
        cudaError_t e = cudaSuccess;
        if (s.cap < T->npix && (e = grow(s, T->npix)) != cudaSuccess) {
            complete(T, MRP_ERR_OOM, cuda_msg("slot buffers", e));
            continue;
        }
        std::string err;
        const Lut* lut = lut_for(w.g, v->params.seed, s.stream, &err);
        if (!lut) { complete(T, MRP_ERR_CUDA, err); continue; }
        s.t = T;
        s.vd = v->dev();
        s.vd.trs = s.trs;
        s.vd.trs_pad = nullptr;   // the slot's own TR levels have no padded or paired copy
        s.vd.mip_tr = nullptr;
        s.vd.pad_pair = nullptr;
        s.vd.lut = lut->d;
        s.vd.lut_dirs = lut->d + kLut * kLut;
        s.vd.gmip0_tex = s.vd.gtr0_tex = s.vd.glut_tex = 0;   // textures: the server's own, below
        for (auto& t : s.vd.gpair_tex) t = 0;
        if (use_tex) {
            if ((e = ensure_tr_textures(s)) != cudaSuccess) {
                complete(T, MRP_ERR_OOM, cuda_msg("slot textures", e));
                release(s);
                continue;
            }
            VolTex* vt = vtex_for(v, s.stream, &err);
            if (!vt) { complete(T, MRP_ERR_CUDA, err); release(s); continue; }
            vt->users++;
            slot_vtex[pick] = vt;
            s.vd.gmip0_tex = vt->mip0.tex;
            s.vd.gtr0_tex = s.gtr0.tex;
            for (int l = 1; l < kGtexPairs; ++l) s.vd.gpair_tex[l] = s.gpair[l].tex;
            s.vd.glut_tex = lut->tex.tex;
        }
        s.view = make_view(v, &w, w.frame_offset, 0);
        HitRecords rec = s.records();
        const GtexLevel* trl = &s.gtr0;
        const float* trsrc = s.trs;
        if ((e = build_tr_levels(s.trs, v->mips, v->mip_occ, w.light_dir, w.alpha, s.stream)) != cudaSuccess ||
            (use_tex && ((e = gtex_fill(&trl, &trsrc, 1, g.sms, s.stream)) != cudaSuccess ||
                         (e = gtex_fill_pairs(s.gpair, v->mips, s.trs, g.sms, s.stream)) != cudaSuccess)) ||
            (e = launch_hit(s.vd, s.view, rec, s.accum, s.stream)) != cudaSuccess ||
            (e = launch_gather_rec(s.vd, s.view, rec, s.feat, cfg.precision != MRP_FP32, s.stream)) != cudaSuccess) {
            complete(T, MRP_ERR_CUDA, cuda_msg("request launch", e));
            release(s);
            continue;
        }
        if (cfg.precision == MRP_FP32) {   // FP32 network per request, no batching
            if ((e = launch_mlp_rec_fp32(s.vd, s.view, rec, s.feat, g.d_weights, s.accum, s.stream)) != cudaSuccess) {
                complete(T, MRP_ERR_CUDA, cuda_msg("network", e));
                release(s);
                continue;
            }
            T->t.features_ms = T->t.network_ms = ms_since(t0);
            enqueue_output(s, false);
        } else {
            cudaEventRecord(s.ev_feat, s.stream);
            s.state = kFeatures;
        }
    }
    if (moved) {
        std::lock_guard<std::mutex> lk(mu);
        stats.bytes_in_use = used;
        if (used > stats.peak_bytes) stats.peak_bytes = used;
    }
    return moved;
}

// One persistent launch over every request whose features are ready.
bool mrp_server::launch_network() {
    if (net_busy) return false;
    batch.clear();
    for (int i = 0; i < (int)slots.size() && (int)batch.size() < kTcMaxSegments; ++i) {
        Slot& s = slots[i];
        if (s.state != kFeatures) continue;
        cudaError_t q = cudaEventQuery(s.ev_feat);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess) {
            complete(s.t, MRP_ERR_CUDA, cuda_msg("features", q));
            release(s);
            continue;
        }
        s.t->t.features_ms = ms_since(t0);
        h_segs[batch.size()] = tc_segment(s.vd, s.view, s.records(), s.feat, s.accum);
        batch.push_back(i);
    }
    if (batch.empty()) return false;
    int n = (int)batch.size();
    cudaError_t e;
    if ((e = cudaMemcpyAsync(d_segs, h_segs, n * sizeof(TcSegment), cudaMemcpyHostToDevice, net)) != cudaSuccess ||
        (e = cudaMemsetAsync(sc.d + 1, 0, sizeof(int), net)) != cudaSuccess ||
        (e = tc_launch_mlp_segments(g.tc, cfg.precision == MRP_FP8, d_segs, n, sc, g.sms, net)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h_err, sc.d + 1, sizeof(int), cudaMemcpyDeviceToHost, net)) != cudaSuccess ||
        (e = cudaEventRecord(ev_net, net)) != cudaSuccess) {
        for (int i : batch) {
            complete(slots[i].t, MRP_ERR_CUDA, cuda_msg("batched network", e));
            release(slots[i]);
        }
        batch.clear();
        return true;
    }
    for (int i : batch) slots[i].state = kNetwork;
    net_busy = true;
    std::lock_guard<std::mutex> lk(mu);
    stats.batches++;
    stats.batched_requests += n;
    if (n > stats.max_batch) stats.max_batch = n;
    return true;
}

bool mrp_server::finish_network() {
    if (!net_busy) return false;
    cudaError_t q = cudaEventQuery(ev_net);
    if (q == cudaErrorNotReady) return false;
    net_busy = false;
    for (int i : batch) {
        Slot& s = slots[i];
        s.t->t.network_ms = ms_since(t0);
        if (q != cudaSuccess || *h_err) {
            complete(s.t, q != cudaSuccess ? MRP_ERR_CUDA : MRP_ERR_TIMEOUT,
                     q != cudaSuccess ? cuda_msg("batched network", q) : "tensor-core MLP: MMA completion wait timed out");
            release(s);
            continue;
        }
        enqueue_output(s, true);
    }
    batch.clear();
    return true;
}

// Result to the caller's buffer on the slot's stream: device and pinned host
// buffers directly, pageable host memory through the slot's pinned staging.
void mrp_server::enqueue_output(Slot& s, bool after_net) {
    const size_t bytes = s.t->npix * sizeof(float4);
    float* out = s.t->req.out_rgba;
    cudaError_t e = cudaSuccess;
    if (after_net) e = cudaStreamWaitEvent(s.stream, ev_net, 0);
    s.staged_out = false;
    if (e == cudaSuccess) {
        if (s.t->req.out_is_device) {
            e = cudaMemcpyAsync(out, s.accum, bytes, cudaMemcpyDeviceToDevice, s.stream);
        } else {
            cudaPointerAttributes at{};
            bool pinned = cudaPointerGetAttributes(&at, out) == cudaSuccess && at.type == cudaMemoryTypeHost;
            cudaGetLastError();
            if (pinned) {
                e = cudaMemcpyAsync(out, s.accum, bytes, cudaMemcpyDeviceToHost, s.stream);
            } else {
                if (s.staging_cap < bytes) {
                    if (s.staging) mrp::host_free_pinned(s.staging);
                    s.staging = nullptr;
                    s.staging_cap = 0;
                    e = mrp::host_malloc_pinned(&s.staging, bytes);
                    if (e == cudaSuccess) s.staging_cap = bytes;
                }
                if (e == cudaSuccess) e = cudaMemcpyAsync(s.staging, s.accum, bytes, cudaMemcpyDeviceToHost, s.stream);
                s.staged_out = true;
            }
        }
    }
    if (e == cudaSuccess) e = cudaEventRecord(s.ev_done, s.stream);
    if (e != cudaSuccess) {
        complete(s.t, MRP_ERR_CUDA, cuda_msg("result copy", e));
        release(s);
        return;
    }
    s.state = kOutput;
}

bool mrp_server::finish_outputs() {
    bool moved = false;
    for (Slot& s : slots) {
        if (s.state != kOutput) continue;
        cudaError_t q = cudaEventQuery(s.ev_done);
        if (q == cudaErrorNotReady) continue;
        moved = true;
        if (q == cudaSuccess && s.staged_out) std::memcpy(s.t->req.out_rgba, s.staging, s.t->npix * sizeof(float4));
        std::shared_ptr<Ticket> T = s.t;
        release(s);
        complete(T, q == cudaSuccess ? MRP_OK : MRP_ERR_CUDA, q == cudaSuccess ? "" : cuda_msg("result copy", q));
    }
    return moved;
}

void mrp_server::run() {
    cudaSetDevice(g.device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            while (!incoming.empty()) {
                pending.push_back(incoming.front());
                incoming.pop_front();
            }
            bool busy = !pending.empty() || net_busy;
            for (const Slot& s : slots) busy = busy || s.state != kFree;
            if (!busy) {
                if (stopping) return;
                cv_work.wait_for(lk, std::chrono::milliseconds(20));
                continue;
            }
        }
        bool moved = finish_outputs();
        moved = finish_network() || moved;
        moved = launch_network() || moved;
        moved = admit() || moved;
        if (!moved) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

extern "C" {

void mrp_serve_default_config(mrp_serve_config* c) {
    if (!c) return;
    c->memory_budget = (size_t)120 << 30;
    c->max_slots = 16;
    c->precision = MRP_BF16;
    c->slot_pixels = 0;
}

mrp_status mrp_serve_open(const mrp_serve_config* cfg_in, mrp_server** out) {
    TRY(need_init());
    if (!out) return fail(MRP_ERR_INVALID, "null argument");
    mrp_serve_config cfg;
    mrp_serve_default_config(&cfg);
    if (cfg_in) cfg = *cfg_in;
    if (cfg.max_slots < 1 || cfg.max_slots > kTcMaxSegments)
        return fail(MRP_ERR_INVALID, "max_slots %d out of range [1, %d]", cfg.max_slots, kTcMaxSegments);
    if (cfg.precision != MRP_FP32 && cfg.precision != MRP_BF16 && cfg.precision != MRP_FP8)
        return fail(MRP_ERR_INVALID, "unknown precision %d", (int)cfg.precision);
    if (cfg.slot_pixels > (1ull << 26)) return fail(MRP_ERR_INVALID, "slot_pixels %zu too large", cfg.slot_pixels);
    if (cfg.slot_pixels && (slot_bytes(cfg.slot_pixels) + kLutBytes + (cfg.precision != MRP_FP32 ? tr_tex_bytes() : 0)) *
                                   (size_t)cfg.max_slots > cfg.memory_budget)
        return fail(MRP_ERR_BUDGET, "%d slots of %zu pixels exceed the budget of %zu bytes", cfg.max_slots,
                    cfg.slot_pixels, cfg.memory_budget);
    std::unique_ptr<mrp_server> S(new mrp_server());
    S->cfg = cfg;
    S->t0 = Clock::now();
    auto cleanup = [&](mrp_status st) {
        mrp_server* p = S.release();
        p->stopping = true;
        for (Slot& s : p->slots) {
            p->free_buffers(s);
            if (s.stream) cudaStreamDestroy(s.stream);
            if (s.ev_feat) cudaEventDestroy(s.ev_feat);
            if (s.ev_done) cudaEventDestroy(s.ev_done);
        }
        if (p->net) cudaStreamDestroy(p->net);
        if (p->ev_net) cudaEventDestroy(p->ev_net);
        tc_free_scratch(p->sc);
        mrp::dev_free(p->d_segs);
        if (p->h_segs) mrp::host_free_pinned(p->h_segs);
        if (p->h_err) mrp::host_free_pinned(p->h_err);
        delete p;
        return st;
    };
    cudaError_t e;
    S->slots.resize(cfg.max_slots);
    S->slot_vtex.assign(cfg.max_slots, nullptr);
    S->tex_mode = cfg.precision != MRP_FP32;
    for (Slot& s : S->slots)
        if ((e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&s.ev_feat, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&s.ev_done, cudaEventDisableTiming)) != cudaSuccess)
            return cleanup(fail(MRP_ERR_CUDA, "slot streams: %s", cudaGetErrorString(e)));
    if ((e = cudaStreamCreateWithFlags(&S->net, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&S->ev_net, cudaEventDisableTiming)) != cudaSuccess ||
        (e = tc_ensure_scratch(S->sc)) != cudaSuccess ||
        (e = mrp::dev_malloc(&S->d_segs, kTcMaxSegments * sizeof(TcSegment))) != cudaSuccess ||
        (e = mrp::host_malloc_pinned(&S->h_segs, kTcMaxSegments * sizeof(TcSegment))) != cudaSuccess ||
        (e = mrp::host_malloc_pinned(&S->h_err, sizeof(int))) != cudaSuccess)
        return cleanup(fail(MRP_ERR_CUDA, "server set-up: %s", cudaGetErrorString(e)));
    *S->h_err = 0;
    {   // keep freed slot memory in the device pool instead of returning it
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, g.device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    if (cfg.slot_pixels) {
        // slots sized at open also get their texture copies now: array
        // allocations are synchronous and would stall the worker mid-stream
        for (Slot& s : S->slots)
            if ((e = S->grow(s, cfg.slot_pixels)) != cudaSuccess ||
                (S->tex_mode && (e = S->ensure_tr_textures(s)) != cudaSuccess))
                return cleanup(fail(MRP_ERR_OOM, "slot buffers: %s", cudaGetErrorString(e)));
        for (Slot& s : S->slots)
            if ((e = cudaStreamSynchronize(s.stream)) != cudaSuccess)
                return cleanup(fail(MRP_ERR_CUDA, "slot buffers: %s", cudaGetErrorString(e)));
        S->stats.peak_bytes = S->stats.bytes_in_use = S->used;
    }
    mrp_server* p = S.release();
    p->worker = std::thread([p] { p->run(); });
    *out = p;
    return MRP_OK;
}

mrp_status mrp_serve_submit(mrp_server* S, const mrp_request* r, uint64_t* ticket) {
    if (!S || !r || !ticket) return fail(MRP_ERR_INVALID, "null argument");
    const mrp_view& w = r->view;
    if (!r->volume || !r->out_rgba) return fail(MRP_ERR_INVALID, "request needs a volume and an output buffer");
    if (!r->volume->has_pyramid) return fail(MRP_ERR_NOT_READY, "volume has no pyramid (call mrp_volume_update)");
    if (w.width <= 0 || w.height <= 0 || (long long)w.width * w.height > (1ll << 26))
        return fail(MRP_ERR_INVALID, "image size %dx%d", w.width, w.height);
    auto T = std::make_shared<Ticket>();
    T->req = *r;
    T->npix = (size_t)w.width * w.height;
    size_t need = slot_bytes(T->npix) + kLutBytes;
    if (S->tex_mode && r->volume->params.gather_filter) need += tr_tex_bytes() + mip_tex_bytes() + kLutTexBytes;
    if (need > S->cfg.memory_budget)
        return fail(MRP_ERR_BUDGET, "request needs %zu bytes, budget is %zu", need, S->cfg.memory_budget);
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) return fail(MRP_ERR_NOT_READY, "server is closing");
    T->id = S->next_id++;
    T->t.submit_ms = ms_since(S->t0);
    S->tickets[T->id] = T;
    S->incoming.push_back(T);
    S->stats.submitted++;
    *ticket = T->id;
    S->cv_work.notify_one();
    return MRP_OK;
}

mrp_status mrp_serve_poll(mrp_server* S, uint64_t ticket, int wait_ms, int* done, mrp_request_timing* timing) {
    if (!S || !done) return fail(MRP_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->tickets.find(ticket);
    if (it == S->tickets.end()) return fail(MRP_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    std::shared_ptr<Ticket> T = it->second;
    if (!T->done && wait_ms != 0) {
        if (wait_ms < 0) S->cv_done.wait(lk, [&] { return T->done; });
        else S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return T->done; });
    }
    *done = T->done ? 1 : 0;
    if (!T->done) return MRP_OK;
    if (timing) *timing = T->t;
    S->tickets.erase(it);
    if (T->status != MRP_OK) return fail(T->status, "%s", T->error.c_str());
    return MRP_OK;
}

mrp_status mrp_serve_stats_get(mrp_server* S, mrp_serve_stats* st) {
    if (!S || !st) return fail(MRP_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    *st = S->stats;
    return MRP_OK;
}

mrp_status mrp_serve_close(mrp_server* S) {
    if (!S) return fail(MRP_ERR_INVALID, "null server");
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
        S->cv_work.notify_all();
    }
    if (S->worker.joinable()) S->worker.join();
    for (Slot& s : S->slots) {
        S->free_buffers(s);
        cudaStreamSynchronize(s.stream);
        if (s.staging) mrp::host_free_pinned(s.staging);
        cudaStreamDestroy(s.stream);
        cudaEventDestroy(s.ev_feat);
        cudaEventDestroy(s.ev_done);
    }
    for (Lut& l : S->luts) {
        gtex_free(&l.tex);
        mrp::dev_free(l.d);
        cudaEventDestroy(l.ready);
    }
    while (!S->vtex.empty()) S->drop_vtex(S->vtex.size() - 1);
    cudaStreamDestroy(S->net);
    cudaEventDestroy(S->ev_net);
    tc_free_scratch(S->sc);
    mrp::dev_free(S->d_segs);
    mrp::host_free_pinned(S->h_segs);
    mrp::host_free_pinned(S->h_err);
    cudaMemPool_t pool;   // give the slots' memory back to the device
    if (cudaDeviceGetDefaultMemPool(&pool, g.device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    delete S;
    return MRP_OK;
}

}  // extern "C"
