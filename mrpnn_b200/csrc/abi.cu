// abi.cu -- host side of the C ABI (include/mrpnn.h): library state, volume
// handles, resource caches and the render loop of VolumeRender::Render.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <dlfcn.h>

#include "abi_internal.h"

using namespace mrp;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string t_err;
namespace mrpi {
Lib g;
mrp_status fail(mrp_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_err = buf;
    return s;
}
}  // namespace mrpi
using namespace mrpi;

// ---------------------------------------------------------------------------
// library state (one device per process)
// ---------------------------------------------------------------------------
namespace {

std::string default_model_path() {
    Dl_info info;
    if (dladdr((void*)&default_model_path, &info) && info.dli_fname) {
        std::string p = info.dli_fname;
        size_t s = p.rfind('/');
        std::string dir = s == std::string::npos ? "." : p.substr(0, s);
        return dir + "/data/mrpnn_model.bin";
    }
    return "mrpnn_model.bin";
}

// Digit permutations of the scrambled radical inverse for bases 2, 3, 5, 7,
// 11: the reference's table (RadicalInversePermutations_, core/volume.cu:1195),
// carried by the model file as HALTON_PERMS; each base's block must be a
// permutation of its digits.
mrp_status halton_perms(const std::map<std::string, std::vector<float>>& m, uint32_t perm[28]) {
    auto it = m.find("HALTON_PERMS");
    if (it == m.end() || it->second.size() != 28) return fail(MRP_ERR_IO, "model file: missing HALTON_PERMS");
    const uint32_t primes[5] = {2, 3, 5, 7, 11}, sums[5] = {0, 2, 5, 10, 17};
    for (int b = 0; b < 5; ++b) {
        uint32_t seen = 0;
        for (uint32_t i = 0; i < primes[b]; ++i) {
            float v = it->second[sums[b] + i];
            if (!(v >= 0.0f && v < (float)primes[b]) || v != (float)(uint32_t)v)
                return fail(MRP_ERR_IO, "model file: HALTON_PERMS is not a digit permutation");
            perm[sums[b] + i] = (uint32_t)v;
            seen |= 1u << perm[sums[b] + i];
        }
        if (seen != (1u << primes[b]) - 1) return fail(MRP_ERR_IO, "model file: HALTON_PERMS is not a digit permutation");
    }
    return MRP_OK;
}

float lerp_h(float a, float b, float v) { return a * (1.0f - v) + b * v; }

// GetSamples23_ (core/vector.cu:304-405): offset and mip layer of stencil
// point i, plus the HG-LUT row v of SetupInputData (core/radiancePredict.cu:458-464).
void stencil_tables(StencilTables& t, const std::vector<float>& dirs) {
    for (int i = 0; i < 192; ++i) {
        float o, layer;
        const float sc = 0.6f;
        if (i < 8) { o = (float)(1.0 / 256.0); o *= lerp_h(sc, 1.0f, 1.0f); layer = 0; }
        else if (i < 16) { o = (float)(2.5 / 256.0); o *= lerp_h(sc, 1.0f, 0.8f); layer = 1; }
        else if (i < 32) { o = (float)(5.5 / 256.0); o *= lerp_h(sc, 1.0f, 0.6f); layer = 2; }
        else if (i < 48) { o = (float)(11.5 / 256.0); o *= lerp_h(sc, 1.0f, 0.4f); layer = 3; }
        else if (i < 64) { o = (float)(23.5 / 256.0); o *= lerp_h(sc, 1.0f, 0.2f); layer = 4; }
        else if (i < 96) { o = (float)(47.5 / 256.0); o *= sc; layer = 5; }
        else if (i < 128) { o = (float)(95.5 / 256.0); o *= sc; layer = 6; }
        else if (i < 160) { o = (float)(191.5 / 256.0); o *= sc; layer = 7; }
        else if (i < 168) { o = (float)(i - 160 + 1); o = (float)(o / 256.0); layer = 0; }
        else if (i < 176) { o = (float)(8.5 + 1 + 2.0 * (i - 168)); o = (float)(o / 256.0); layer = 1; }
        else if (i < 184) { o = (float)(26.5 + 4.0 * (i - 176)); o = (float)(o / 256.0); layer = 2; }
        else { o = (float)(60.5 + 8.0 * (i - 184)); o = (float)(o / 256.0); layer = 3; }
        layer += 0.1f;
        int l = (int)layer;
        t.offset[i] = o;
        t.layer[i] = l;
        float radius = (float)(1 << l) / 256.0f;
        float angle = std::atan(0.5f * radius / o);
        t.lut_v[i] = angle / (3.1415926535f * 60.0f / 180.0f);
    }
    std::memcpy(t.dirs, dirs.data(), sizeof t.dirs);
}

mrp_status read_model(const char* path, std::map<std::string, std::vector<float>>& out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(MRP_ERR_IO, "cannot open model file %s", path);
    char magic[8];
    uint32_t count = 0;
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "MRPNNMD1", 8) != 0 || std::fread(&count, 4, 1, f) != 1) {
        std::fclose(f);
        return fail(MRP_ERR_IO, "%s: not an MRPNN model file", path);
    }
    out.clear();
    for (uint32_t k = 0; k < count; ++k) {
        uint16_t len = 0;
        uint32_t n = 0;
        std::string name;
        if (std::fread(&len, 2, 1, f) != 1) break;
        name.resize(len);
        if (std::fread(&name[0], 1, len, f) != len || std::fread(&n, 4, 1, f) != 1 || n > (1u << 24)) break;
        std::vector<float> v(n);
        if (std::fread(v.data(), 4, n, f) != n) break;
        out[name] = std::move(v);
    }
    std::fclose(f);
    if (out.size() != count) return fail(MRP_ERR_IO, "%s: truncated model file", path);
    return MRP_OK;
}

// Packs the named tensors into the kernel layout (common.cuh).
mrp_status pack_weights(const std::map<std::string, std::vector<float>>& m, std::vector<float>& w) {
    w.clear();
    auto put = [&](const std::string& name, size_t n) -> bool {
        auto it = m.find(name);
        if (it == m.end() || it->second.size() != n) { t_err = "model tensor " + name + " missing or mis-sized"; return false; }
        w.insert(w.end(), it->second.begin(), it->second.end());
        return true;
    };
    auto block = [&](const std::string& se, const std::string& d, const std::string& tr, const std::string& hg,
                     int wdt) -> bool {
        return put(se + "1W", 64) && put(se + "2W", 24) && put(d + "W", wdt * wdt) && put(d + "B", wdt) &&
               put(tr + "W", wdt * wdt) && put(tr + "B", wdt) && put(hg + "W", wdt * wdt) && put(hg + "B", wdt);
    };
    for (int k = 0; k < 8; ++k) {
        std::string s = std::to_string(k);
        if (!block("LSE" + s, "L" + s + "1", "L_Tr" + s + "1", "L_Hg" + s + "1", kMainW[k])) return MRP_ERR_IO;
    }
    if (!(put("L81W", 1024) && put("L81B", 32) && put("L_Tr81W", 1024) && put("L_Tr81B", 32) && put("L_Hg81W", 1024) &&
          put("L_Hg81B", 32)))
        return MRP_ERR_IO;
    for (int k = 0; k < 4; ++k) {
        std::string s = std::to_string(k);
        if (!block("LDSE" + s, "LD" + s + "1", "LD_Tr" + s + "1", "LD_Hg" + s + "1", 8)) return MRP_ERR_IO;
    }
    if (!(put("LD41W", 64) && put("LD41B", 8) && put("LD_Tr41W", 64) && put("LD_Tr41B", 8) && put("LD_Hg41W", 64) &&
          put("LD_Hg41B", 8)))
        return MRP_ERR_IO;
    if (!(put("LGGSW", 24) && put("LGGSB", 8) && put("LSEFin1W", 1200) && put("LSEFin2W", 96) && put("LC0W", 16384) &&
          put("LC0B", 128) && put("LC1W", 8192) && put("LC1B", 64) && put("LC2W", 2048) && put("LC2B", 32) &&
          put("LXW", 512) && put("LXB", 16)))
        return MRP_ERR_IO;
    for (int k = 0; k < 12; ++k)
        if (!(put("LX" + std::to_string(k) + "W", 256) && put("LX" + std::to_string(k) + "B", 16))) return MRP_ERR_IO;
    if (!(put("LX12W", 16) && put("LX12B", 1))) return MRP_ERR_IO;
    if ((int)w.size() != kWeightCount) return fail(MRP_ERR_IO, "packed %zu weights, expected %d", w.size(), kWeightCount);
    return MRP_OK;
}

mrp_status ensure_scratch(size_t bytes) {
    if (g.scratch_bytes >= bytes) return MRP_OK;
    if (g.scratch) mrp::dev_free(g.scratch);
    g.scratch = nullptr;
    g.scratch_bytes = 0;
    CU(mrp::dev_malloc(&g.scratch, bytes));
    g.scratch_bytes = bytes;
    return MRP_OK;
}

}  // namespace

namespace mrp {
std::atomic<unsigned long long> g_alloc_calls{0};
}

extern "C" {

const char* mrp_last_error(void) { return t_err.c_str(); }
const char* mrp_version(void) { return "mrpnn_b200 0.1 (sm_100a)"; }
unsigned long long mrp_debug_alloc_calls(void) { return mrp::g_alloc_calls.load(); }

void mrp_default_params(mrp_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->scatter_rate[0] = p->scatter_rate[1] = p->scatter_rate[2] = 1.001f;
    p->tr_scale = 1.0f;
    p->env_exp = 1.0f;
    p->bake_res = 768;
    p->bake_replicate_seeding = 1;
    p->precision = MRP_FP32;
    p->seed = 0;
    p->gather_filter = 1;
}

mrp_status mrp_load_model(const char* path) {
    std::lock_guard<std::mutex> lk(g.mu);
    if (!g.ready) return fail(MRP_ERR_NOT_READY, "mrp_init has not been called");
    std::map<std::string, std::vector<float>> m;
    TRY(read_model(path, m));
    std::vector<float> w;
    if (pack_weights(m, w) != MRP_OK) return fail(MRP_ERR_IO, "%s: %s", path, t_err.c_str());
    auto it = m.find("STENCIL_DIRS");
    if (it == m.end() || it->second.size() != 480) return fail(MRP_ERR_IO, "%s: missing STENCIL_DIRS", path);
    StencilTables st;
    stencil_tables(st, it->second);
    uint32_t perm[28];
    if (halton_perms(m, perm) != MRP_OK) return fail(MRP_ERR_IO, "%s: %s", path, t_err.c_str());
    CU(set_stencil_tables(st));
    CU(set_halton_permutations(perm));
    std::vector<float> wd(kWeightCountDev, 0.0f);
    std::copy(w.begin(), w.end(), wd.begin());
    for (int j = 0; j < 128; ++j)
        for (int o = 0; o < 64; ++o) wd[kLC1T + j * 64 + o] = w[kLC1W + o * 128 + j];
    for (int j = 0; j < 75; ++j)
        for (int o = 0; o < 16; ++o) wd[kFin1T + j * 16 + o] = w[kLSEFin1W + o * 75 + j];
    if (!g.d_weights) CU(mrp::dev_malloc(&g.d_weights, sizeof(float) * kWeightCountDev));
    CU(cudaMemcpy(g.d_weights, wd.data(), sizeof(float) * kWeightCountDev, cudaMemcpyHostToDevice));
    CU(tc_prepare_weights(w.data(), g.tc));
    g.tc.d_fp32 = g.d_weights;
    g.model = std::move(m);
    g.h_weights = std::move(w);
    return MRP_OK;
}

mrp_status mrp_init(int device, const char* model_path) {
    {
        std::lock_guard<std::mutex> lk(g.mu);
        if (!g.ready) {
            int n = 0;
            cudaError_t e = cudaGetDeviceCount(&n);
            if (e != cudaSuccess || n == 0)
                return fail(MRP_ERR_NO_DEVICE, "no CUDA device (%s)", cudaGetErrorString(e));
            if (device < 0 || device >= n) return fail(MRP_ERR_INVALID, "device %d out of range (%d)", device, n);
            CU(cudaSetDevice(device));
            cudaDeviceProp prop;
            CU(cudaGetDeviceProperties(&prop, device));
            if (prop.major != 10)
                return fail(MRP_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a", device,
                            prop.major, prop.minor);
            g.device = device;
            g.sms = prop.multiProcessorCount;
            CU(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
            g.ready = true;
        } else {
            CU(cudaSetDevice(g.device));
        }
    }
    if (g.d_weights && !model_path) return MRP_OK;
    std::string p = model_path ? model_path : default_model_path();
    return mrp_load_model(p.c_str());
}

mrp_status mrp_volume_create(int res, mrp_volume** out) { return mrp_volume_create_ex(res, MRP_STORAGE_FP32, out); }

mrp_status mrp_volume_create_ex(int res, mrp_storage storage, mrp_volume** out) {
    TRY(need_init());
    if (!out || res < 2 || res > 2048) return fail(MRP_ERR_INVALID, "volume resolution %d out of range [2, 2048]", res);
    if (storage != MRP_STORAGE_FP32 && storage != MRP_STORAGE_FP16)
        return fail(MRP_ERR_INVALID, "unknown density storage %d", (int)storage);
    mrp_volume* v = new mrp_volume();
    static std::atomic<uint64_t> next_uid{1};
    v->uid = next_uid.fetch_add(1);
    v->res = res;
    mrp_default_params(&v->params);
    auto cleanup = [&](mrp_status s) { mrp_volume_destroy(v); return s; };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&v->ev0)) != cudaSuccess || (e = cudaEventCreate(&v->ev1)) != cudaSuccess ||
        (e = cudaEventCreate(&v->ev_stage[0])) != cudaSuccess || (e = cudaEventCreate(&v->ev_stage[1])) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&v->stream_copy, cudaStreamNonBlocking)) != cudaSuccess)
        return cleanup(fail(MRP_ERR_CUDA, "stream/event: %s", cudaGetErrorString(e)));
    for (int s = 0; s < 2; ++s)
        if ((e = cudaEventCreateWithFlags(&v->ev_done[s], cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&v->ev_copied[s], cudaEventDisableTiming)) != cudaSuccess)
            return cleanup(fail(MRP_ERR_CUDA, "event: %s", cudaGetErrorString(e)));
    size_t n = (size_t)res * res * res;
    v->occ_res = (res + (1 << v->occ_shift) - 1) >> v->occ_shift;
    v->occ2_res = (v->occ_res + 3) / 4;
    size_t nocc = (size_t)v->occ_res * v->occ_res * v->occ_res;
    if ((storage == MRP_STORAGE_FP16 ? (e = mrp::dev_malloc(&v->density_h, n * sizeof(__half)))
                                     : (e = mrp::dev_malloc(&v->density, n * sizeof(float)))) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->mips, kMipFloats * sizeof(float))) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->trs, kTrFloats * sizeof(float))) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->lut, kLutAlloc * sizeof(float))) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->occ, nocc)) != cudaSuccess || (e = mrp::dev_malloc(&v->mip_occ, kMipOccBytes)) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->occ2, (size_t)v->occ2_res * v->occ2_res * v->occ2_res)) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->d_maxbits, sizeof(int))) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->d_bounds, 6 * sizeof(int))) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->mips_pad, kPadLevelFloats * sizeof(float))) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->trs_pad, kPadLevelFloats * sizeof(float))) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->mip_tr, mip_tr_offset(5) * sizeof(float2))) != cudaSuccess ||
        (e = mrp::dev_malloc(&v->pad_pair, kPadLevelFloats * sizeof(float2))) != cudaSuccess)
        return cleanup(fail(e == cudaErrorMemoryAllocation ? MRP_ERR_OOM : MRP_ERR_CUDA, "volume allocation: %s",
                            cudaGetErrorString(e)));
    if (v->density_h) cudaMemsetAsync(v->density_h, 0, n * sizeof(__half), v->stream);
    else cudaMemsetAsync(v->density, 0, n * sizeof(float), v->stream);
    *out = v;
    return MRP_OK;
}

static void drop_density_texture(mrp_volume* v);
static void drop_gather_textures(mrp_volume* v);

mrp_status mrp_volume_destroy(mrp_volume* v) {
    if (!v) return MRP_OK;
    if (v->stream) cudaStreamSynchronize(v->stream);
    if (v->stream_copy) cudaStreamSynchronize(v->stream_copy);
    mrp::dev_free(v->accum_alt);
    mrp::dev_free(v->density); mrp::dev_free(v->density_h); mrp::dev_free(v->mips); mrp::dev_free(v->trs); mrp::dev_free(v->lut); mrp::dev_free(v->baked);
    mrp::dev_free(v->occ); mrp::dev_free(v->occ2); mrp::dev_free(v->mip_occ); mrp::dev_free(v->d_maxbits); mrp::dev_free(v->d_bounds); mrp::dev_free(v->mips_pad); mrp::dev_free(v->trs_pad); mrp::dev_free(v->mip_tr); mrp::dev_free(v->pad_pair); mrp::dev_free(v->accum); mrp::dev_free(v->sum3); mrp::dev_free(v->first_pos);
    mrp::dev_free(v->counter);
    mrp::dev_free(v->hdri);
    drop_density_texture(v);
    drop_gather_textures(v);
    gtex_free(&v->baked_gtex);
    mrp::dev_free(v->rec_count); mrp::dev_free(v->rec_pix); mrp::dev_free(v->rec_f); mrp::dev_free(v->feat);
    tc_free_scratch(v->tc);
    free_multiview(v);
    if (v->ev0) cudaEventDestroy(v->ev0);
    if (v->ev1) cudaEventDestroy(v->ev1);
    for (auto& ev : v->ev_stage) if (ev) cudaEventDestroy(ev);
    for (int s = 0; s < 2; ++s) {
        if (v->ev_done[s]) cudaEventDestroy(v->ev_done[s]);
        if (v->ev_copied[s]) cudaEventDestroy(v->ev_copied[s]);
    }
    if (v->stream_copy) cudaStreamDestroy(v->stream_copy);
    if (v->stream) cudaStreamDestroy(v->stream);
    delete v;
    return MRP_OK;
}

static void drop_density_texture(mrp_volume* v) {
    if (v->dens_tex) cudaDestroyTextureObject(v->dens_tex);
    if (v->dens_arr) mrp::dev_free_array(v->dens_arr);
    v->dens_tex = 0;
    v->dens_arr = nullptr;
}

// The density grid copied into a 3D array (width = z, the fastest axis, as
// the reference's texture coordinate x = z) behind a trilinear texture with
// border addressing and normalized coordinates, as Update binds
// _DensityVolume (core/volume.cu:1458-1465).
static mrp_status ensure_density_texture(mrp_volume* v) {
    if (v->dens_tex) return MRP_OK;
    const int R = v->res;
    cudaChannelFormatDesc desc = v->density_h ? cudaCreateChannelDescHalf() : cudaCreateChannelDesc<float>();
    const cudaExtent ext = make_cudaExtent(R, R, R);
    CU(mrp::dev_malloc_3d_array(&v->dens_arr, &desc, ext));
    cudaMemcpy3DParms cp = {};
    const size_t elem = v->density_h ? sizeof(__half) : sizeof(float);
    cp.srcPtr = make_cudaPitchedPtr(v->density_h ? (void*)v->density_h : (void*)v->density, R * elem, R, R);
    cp.dstArray = v->dens_arr;
    cp.extent = ext;
    cp.kind = cudaMemcpyDeviceToDevice;
    cudaError_t e = cudaMemcpy3DAsync(&cp, v->stream);
    cudaResourceDesc res = {};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = v->dens_arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    if (e == cudaSuccess) e = cudaCreateTextureObject(&v->dens_tex, &res, &td, nullptr);
    if (e != cudaSuccess) {
        drop_density_texture(v);
        CU(e);
    }
    return MRP_OK;
}

static void drop_gather_textures(mrp_volume* v) {
    gtex_free(&v->gmip0);
    gtex_free(&v->gtr0);
    for (auto& L : v->gpair) gtex_free(&L);
    gtex_free(&v->glut);
    v->gtex_alloc = false;
    v->gtex_dirty = 7;
}

// The gather's textures, bound as the reference binds Mip(i), TR_Mip(i) and
// _HGLut (gather_tex.cu): allocated the first time a BF16 / FP8 gather with
// gather_filter asks for them, then refreshed on the volume's stream from
// the linear copies that the builders rewrote.  Called after the LUT and TR
// levels are current.
static mrp_status sync_gather_textures(mrp_volume* v) {
    if (!v->gather_tex_wanted() || !v->has_pyramid || !v->has_tr || !v->has_lut) return MRP_OK;
    if (!v->gtex_alloc) {
        cudaError_t e = cudaSuccess;
        e = gtex_alloc_level(256, false, &v->gmip0);
        if (e == cudaSuccess) e = gtex_alloc_level(128, true, &v->gtr0);
        for (int l = 1; l < kGtexPairs && e == cudaSuccess; ++l) e = gtex_alloc_pair(256 >> l, &v->gpair[l]);
        if (e == cudaSuccess) e = gtex_alloc_lut(&v->glut);
        if (e != cudaSuccess) {
            drop_gather_textures(v);
            CU(e);
        }
        v->gtex_alloc = true;
        v->gtex_dirty = 7;
    }
    const GtexLevel* lv[3];
    const float* src[3];
    int k = 0;
    if (v->gtex_dirty & 1) { lv[k] = &v->gmip0; src[k] = v->mips; ++k; }
    if (v->gtex_dirty & 2) { lv[k] = &v->gtr0; src[k] = v->trs; ++k; }
    if (v->gtex_dirty & 4) { lv[k] = &v->glut; src[k] = v->lut; ++k; }
    if (k) CU(gtex_fill(lv, src, k, g.sms, v->stream));
    if (v->gtex_dirty & 3) CU(gtex_fill_pairs(v->gpair, v->mips, v->trs, g.sms, v->stream));
    v->gtex_dirty = 0;
    return MRP_OK;
}

// The baked NEE grid copied into an fp16 3D array behind a trilinear
// texture with clamp addressing, as Update_CachedTR binds TR_Mip(0) to the
// baked array (core/volume.cu:1687-1693), for the tracer's NEE lookup under
// tracer_filter; refilled after every bake.
static mrp_status ensure_baked_texture(mrp_volume* v) {
    if (v->baked_gtex.arr && v->baked_gtex.n != v->bk_res) {
        CU(cudaStreamSynchronize(v->stream));   // arrays are not stream-ordered
        gtex_free(&v->baked_gtex);
        v->baked_gtex_ok = false;
    }
    if (!v->baked_gtex.arr) {
        CU(gtex_alloc_level(v->bk_res, true, &v->baked_gtex));
        v->baked_gtex_ok = false;
    }
    if (!v->baked_gtex_ok) {
        const GtexLevel* lv = &v->baked_gtex;
        const float* src = v->baked;
        CU(gtex_fill(&lv, &src, 1, g.sms, v->stream));
        v->baked_gtex_ok = true;
    }
    return MRP_OK;
}

static void invalidate(mrp_volume* v) {
    drop_density_texture(v);
    v->has_pyramid = v->has_tr = v->has_baked = false;
    v->has_bounds = false;
    v->tr_alpha = NAN; v->bk_alpha = NAN;
}

mrp_status mrp_volume_set_data(mrp_volume* v, const float* data, int res, int is_device) {
    TRY(need_init());
    if (!v || !data || res != v->res) return fail(MRP_ERR_INVALID, "set_data: resolution %d != volume %d", res, v ? v->res : -1);
    size_t n = (size_t)res * res * res;
    if (!v->density_h) {
        CU(cudaMemcpyAsync(v->density, data, n * sizeof(float), is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           v->stream));
    } else if (is_device) {
        CU(launch_narrow(data, n, v->density_h, g.sms, v->stream));
    } else {
        // fp16 storage from host floats: through a device staging buffer of
        // at most 16 Mi floats, rounded on the device
        const size_t chunk = std::min<size_t>(n, (size_t)16 << 20);
        float* stage = nullptr;
        CU(mrp::dev_malloc(&stage, chunk * sizeof(float)));
        cudaError_t e = cudaSuccess;
        for (size_t i = 0; i < n && e == cudaSuccess; i += chunk) {
            const size_t m = std::min(chunk, n - i);
            e = cudaMemcpyAsync(stage, data + i, m * sizeof(float), cudaMemcpyHostToDevice, v->stream);
            if (e == cudaSuccess) e = launch_narrow(stage, m, v->density_h + i, g.sms, v->stream);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
        mrp::dev_free(stage);
        CU(e);
    }
    CU(cudaStreamSynchronize(v->stream));
    v->has_data = true;
    invalidate(v);
    return MRP_OK;
}

mrp_status mrp_volume_fill(mrp_volume* v, mrp_fill_fn fn, void* user) {
    TRY(need_init());
    if (!v || !fn) return fail(MRP_ERR_INVALID, "fill: null argument");
    int R = v->res;
    std::vector<float> host((size_t)R * R * R);
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (int i = (int)t; i < R; i += (int)nt)
                for (int j = 0; j < R; ++j)
                    for (int k = 0; k < R; ++k) {
                        float u = (float)((i + 0.5) / R), w2 = (float)((j + 0.5) / R), w3 = (float)((k + 0.5) / R);
                        host[((size_t)i * R + j) * R + k] = fn(i, j, k, u, w2, w3, user);
                    }
        });
    for (auto& t : th) t.join();
    return mrp_volume_set_data(v, host.data(), R, 0);
}

mrp_status mrp_volume_generate_fbm(mrp_volume* v, uint32_t seed, float base_freq, int octaves, float gain) {
    TRY(need_init());
    if (!v || octaves < 1 || octaves > 16) return fail(MRP_ERR_INVALID, "fbm: bad arguments");
    if (v->density_h) CU(launch_fbm(v->density_h, v->res, seed, base_freq, octaves, gain, g.sms, v->stream));
    else CU(launch_fbm(v->density, v->res, seed, base_freq, octaves, gain, g.sms, v->stream));
    CU(cudaStreamSynchronize(v->stream));
    v->has_data = true;
    invalidate(v);
    return MRP_OK;
}

mrp_status mrp_volume_set_max_density(mrp_volume* v, float md) {
    if (!v || !(md > 0)) return fail(MRP_ERR_INVALID, "max density must be > 0");
    v->max_density = md;
    v->max_override = true;
    v->has_baked = false; v->bk_alpha = NAN;
    return MRP_OK;
}

mrp_status mrp_volume_update(mrp_volume* v, int process_mips) {
    TRY(need_init());
    if (!v) return fail(MRP_ERR_INVALID, "null volume");
    if (!v->has_data) return fail(MRP_ERR_NOT_READY, "update: no data set");
    int R = v->res;
    size_t n = (size_t)R * R * R;
    if (!v->max_override) {
        int init;
        { float f0 = 0.00001f; std::memcpy(&init, &f0, sizeof init); }
        CU(cudaMemcpyAsync(v->d_maxbits, &init, sizeof(int), cudaMemcpyHostToDevice, v->stream));
        if (v->density_h) CU(launch_max_density(v->density_h, n, v->d_maxbits, g.sms, v->stream));
        else CU(launch_max_density(v->density, n, v->d_maxbits, g.sms, v->stream));
        int bits = 0;
        CU(cudaMemcpyAsync(&bits, v->d_maxbits, sizeof(int), cudaMemcpyDeviceToHost, v->stream));
        CU(cudaStreamSynchronize(v->stream));
        std::memcpy(&v->max_density, &bits, sizeof(float));
    }
    if (v->density_h) CU(launch_occupancy(v->density_h, R, v->occ_shift, v->occ_res, v->occ, g.sms, v->stream));
    else CU(launch_occupancy(v->density, R, v->occ_shift, v->occ_res, v->occ, g.sms, v->stream));
    CU(launch_occupancy_coarse(v->occ, v->occ_res, v->occ2, g.sms, v->stream));
    {
        const int init[6] = {R, R, R, -1, -1, -1};
        CU(cudaMemcpyAsync(v->d_bounds, init, sizeof init, cudaMemcpyHostToDevice, v->stream));
        if (v->density_h) CU(launch_nonzero_bounds(v->density_h, R, v->d_bounds, g.sms, v->stream));
        else CU(launch_nonzero_bounds(v->density, R, v->d_bounds, g.sms, v->stream));
        CU(cudaMemcpyAsync(v->nz_bounds, v->d_bounds, sizeof v->nz_bounds, cudaMemcpyDeviceToHost, v->stream));
        CU(cudaStreamSynchronize(v->stream));
        v->has_bounds = true;
    }
    if (process_mips) {
        // core/volume.cu:1476-1514: halve to the largest power of two >= 256
        // below the input, then 9 levels 256 >> m, each from the previous one.
        int res = 256;
        while (res * 2 < R) res <<= 1;
        // (the first level reads the density grid in its storage type; every
        // level after it is fp32)
        const float* src = v->density;
        int src_res = R;
        float* tmp[2] = {nullptr, nullptr};
        int which = 0;
        auto resample = [&](float* dst, int r) {
            return src == nullptr && v->density_h ? launch_resample(dst, r, v->density_h, src_res, g.sms, v->stream)
                                                  : launch_resample(dst, r, src, src_res, g.sms, v->stream);
        };
        for (; res > 256; res >>= 1) {
            float*& t = tmp[which];
            if (!t) CU(mrp::dev_malloc(&t, (size_t)res * res * res * sizeof(float)));
            CU(resample(t, res));
            src = t;
            src_res = res;
            which ^= 1;
        }
        for (int m = 0; m < 9; ++m) {
            int r = 256 >> m;
            float* dst = v->mips + mip_offset(m);
            CU(resample(dst, r));
            src = dst;
            src_res = r;
        }
        for (int m = 0; m < kOccMips; ++m)
            CU(launch_occupancy(v->mips + mip_offset(m), 256 >> m, 3, 32 >> m, v->mip_occ + mip_occ_offset(m), g.sms,
                                v->stream));
        CU(launch_pad_levels(v->mips + mip_offset(5), v->mips + mip_offset(6), v->mips + mip_offset(7), false,
                             v->mips_pad, v->stream));
        CU(cudaStreamSynchronize(v->stream));
        mrp::dev_free(tmp[0]);
        mrp::dev_free(tmp[1]);
        v->has_pyramid = true;
        v->gtex_dirty |= 1;
        ++v->pyramid_version;
    }
    CU(cudaStreamSynchronize(v->stream));
    v->has_tr = false; v->tr_alpha = NAN;
    v->has_baked = false; v->bk_alpha = NAN;
    return MRP_OK;
}

mrp_status mrp_volume_get_info(const mrp_volume* v, mrp_volume_info* info) {
    if (!v || !info) return fail(MRP_ERR_INVALID, "null argument");
    std::memset(info, 0, sizeof *info);
    info->res = v->res;
    info->max_density = v->max_density;
    info->has_pyramid = v->has_pyramid;
    info->has_lut = v->has_lut;
    info->has_tr = v->has_tr;
    info->has_baked_tr = v->has_baked;
    info->lut_g = v->lut_g;
    info->tr_alpha = v->tr_alpha;
    for (int i = 0; i < 3; ++i) info->tr_light[i] = v->tr_light[i];
    size_t R = v->res;
    info->device_bytes = R * R * R * (v->density_h ? 2 : 4) + kMipFloats * 4 + kTrFloats * 4 + kLut * kLut * 4 +
                         (size_t)v->baked_alloc_res * v->baked_alloc_res * v->baked_alloc_res * 4;
    return MRP_OK;
}

mrp_status mrp_set_params(mrp_volume* v, const mrp_params* p) {
    if (!v || !p) return fail(MRP_ERR_INVALID, "null argument");
    if (p->bake_res < 2 || p->bake_res > 2048) return fail(MRP_ERR_INVALID, "bake_res %d out of range", p->bake_res);
    if (p->precision != MRP_FP32 && p->precision != MRP_BF16 && p->precision != MRP_FP8)
        return fail(MRP_ERR_INVALID, "unknown precision %d", (int)p->precision);
    if (p->nee_mode != 0 && p->nee_mode != 1) return fail(MRP_ERR_INVALID, "nee_mode %d (0 or 1)", p->nee_mode);
    if (p->gather_filter != 0 && p->gather_filter != 1)
        return fail(MRP_ERR_INVALID, "gather_filter %d (0 or 1)", p->gather_filter);
    bool bake_changed = p->bake_res != v->params.bake_res || p->tr_scale != v->params.tr_scale ||
                        p->bake_replicate_seeding != v->params.bake_replicate_seeding || p->seed != v->params.seed;
    bool lut_changed = p->seed != v->params.seed;
    v->params = *p;
    if (bake_changed) { v->has_baked = false; v->bk_alpha = NAN; }
    if (lut_changed) { v->has_lut = false; v->lut_g = NAN; }
    return MRP_OK;
}
mrp_status mrp_get_params(const mrp_volume* v, mrp_params* p) {
    if (!v || !p) return fail(MRP_ERR_INVALID, "null argument");
    *p = v->params;
    return MRP_OK;
}

mrp_status mrp_hg_lut_lookup(const float* lut, float cos_theta, float angle, float* out) {
    if (!lut || !out) return fail(MRP_ERR_INVALID, "null argument");
    // GetHGLut's own arithmetic: u, v from double expressions, texels clamped
    // to the table, then lerp(a00, a10, frac(v*N)), lerp(a01, a11, frac(v*N))
    // and a lerp of the two by frac(u*N) (core/volume.cu:1424-1442)
    const int N = 512;
    auto lerp = [](float a, float b, float w) { return a * (1.0f - w) + b * w; };
    auto frac = [](float f) { return f - (float)(long)f; };
    auto clampi = [N](int i) { return std::max(std::min(i, N - 1), 0); };
    float u = (float)((double)cos_theta * 0.5 + 0.5);
    float v = (float)((double)angle / (3.1415926535 * 60.0 / 180.0));
    float uN = u * (float)N, vN = v * (float)N;
    int u0 = clampi((int)uN), v0 = clampi((int)vN), u1 = clampi((int)uN + 1), v1 = clampi((int)vN + 1);
    float a00 = lut[u0 + v0 * N], a10 = lut[u1 + v0 * N], a01 = lut[u0 + v1 * N], a11 = lut[u1 + v1 * N];
    float ax0 = lerp(a00, a10, frac(vN));
    float ax1 = lerp(a01, a11, frac(vN));
    *out = lerp(ax0, ax1, frac(uN));
    return MRP_OK;
}

mrp_status mrp_volume_read(mrp_volume* v, mrp_resource which, int level, float* dst, size_t* count, int dst_is_device) {
    if (!v) return fail(MRP_ERR_INVALID, "null volume");
    const void* src = nullptr;
    size_t n = 0, esize = sizeof(float);
    switch (which) {
        case MRP_RES_DENSITY: src = v->density; n = (size_t)v->res * v->res * v->res; break;   // fp16: below
        case MRP_RES_MIP:
            if (level < 0 || level > 8) return fail(MRP_ERR_INVALID, "mip level %d", level);
            src = v->mips + mip_offset(level); n = (size_t)(256 >> level) * (256 >> level) * (256 >> level); break;
        case MRP_RES_TR:
            if (level < 0 || level > 7) return fail(MRP_ERR_INVALID, "TR level %d", level);
            src = v->trs + tr_offset(level); n = (size_t)(128 >> level) * (128 >> level) * (128 >> level); break;
        case MRP_RES_LUT: src = v->lut; n = kLut * kLut; break;
        case MRP_RES_BAKED_TR:
            if (!v->baked) return fail(MRP_ERR_NOT_READY, "no baked TR");
            src = v->baked; n = (size_t)v->bk_res * v->bk_res * v->bk_res; break;
        case MRP_RES_OCCUPANCY: src = v->occ; n = (size_t)v->occ_res * v->occ_res * v->occ_res; esize = 1; break;
        default: return fail(MRP_ERR_INVALID, "unknown resource %d", (int)which);
    }
    if (count) *count = n;
    if (!dst) return MRP_OK;
    if (which == MRP_RES_DENSITY && v->density_h) {   // fp16 storage, widened to the caller's floats
        if (dst_is_device) {
            CU(launch_widen(v->density_h, n, dst, g.sms, v->stream));
        } else {
            const size_t chunk = std::min<size_t>(n, (size_t)16 << 20);
            float* stage = nullptr;
            CU(mrp::dev_malloc(&stage, chunk * sizeof(float)));
            cudaError_t e = cudaSuccess;
            for (size_t i = 0; i < n && e == cudaSuccess; i += chunk) {
                const size_t m = std::min(chunk, n - i);
                e = launch_widen(v->density_h + i, m, stage, g.sms, v->stream);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(dst + i, stage, m * sizeof(float), cudaMemcpyDeviceToHost, v->stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
            }
            mrp::dev_free(stage);
            CU(e);
        }
        CU(cudaStreamSynchronize(v->stream));
        return MRP_OK;
    }
    CU(cudaMemcpyAsync(dst, src, n * esize, dst_is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, v->stream));
    CU(cudaStreamSynchronize(v->stream));
    return MRP_OK;
}

// --- caches ----------------------------------------------------------------
}  // extern "C"
namespace mrpi {
// Fill_TR for all 8 TR levels: level lv (res 128 >> lv) through density mip
// lv + 1 with alpha / 1.73^(lv + 1) (core/volume.cu:1535-1560).
cudaError_t build_tr_levels(float* trs, const float* mips, const uint8_t* mip_occ, const float L[3], float alpha,
                            cudaStream_t s) {
    for (int lv = 0; lv < 8; ++lv) {
        float a = alpha / std::pow(1.73f, (float)lv + 1.0f);
        const uint8_t* occ = mip_occ && lv + 1 < kOccMips ? mip_occ + mip_occ_offset(lv + 1) : nullptr;
        cudaError_t e = launch_tr_level(trs + tr_offset(lv), 128 >> lv, mips + mip_offset(lv + 1), occ, a, L, g.sms, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
}  // namespace mrpi
extern "C" {
}  // extern "C"
namespace mrpi {
mrp_status update_lut_async(mrp_volume* v, float g_) {
    if (v->has_lut && v->lut_g == g_ && v->lut_seed == v->params.seed) return MRP_OK;
    CU(launch_hg_lut(v->lut, g_, v->params.seed, v->stream));
    CU(launch_lut_dirs(v->lut, v->lut + kLut * kLut, v->stream));
    v->gtex_dirty |= 4;
    v->has_lut = true;
    v->lut_g = g_;
    v->lut_seed = v->params.seed;
    return MRP_OK;
}
mrp_status update_tr_async(mrp_volume* v, const float L[3], float alpha) {
    if (!v->has_pyramid) return fail(MRP_ERR_NOT_READY, "TR mips need the pyramid (call mrp_volume_update)");
    if (v->has_tr && v->tr_alpha == alpha && v->tr_light[0] == L[0] && v->tr_light[1] == L[1] && v->tr_light[2] == L[2])
        return sync_gather_textures(v);
    CU(build_tr_levels(v->trs, v->mips, v->mip_occ, L, alpha, v->stream));
    CU(launch_pad_levels(v->trs + tr_offset(4), v->trs + tr_offset(5), v->trs + tr_offset(6), true, v->trs_pad,
                         v->stream));
    CU(launch_interleave_mip_tr(v->mips, v->trs, v->mip_tr, g.sms, v->stream));
    CU(launch_pair_padded(v->mips_pad, v->trs_pad, v->pad_pair, v->stream));
    v->has_tr = true;
    v->tr_alpha = alpha;
    std::memcpy(v->tr_light, L, sizeof v->tr_light);
    v->gtex_dirty |= 2;
    return sync_gather_textures(v);
}
}  // namespace mrpi
extern "C" {
}  // extern "C"
namespace mrpi {
mrp_status update_baked_async(mrp_volume* v, const float L[3], float alpha) {
    int B = v->params.bake_res;
    if (v->has_baked && v->bk_alpha == alpha && v->bk_res == B && v->bk_seed == v->params.seed &&
        v->bk_light[0] == L[0] && v->bk_light[1] == L[1] && v->bk_light[2] == L[2])
        return MRP_OK;
    if (v->baked_alloc_res != B) {
        mrp::dev_free(v->baked);
        v->baked = nullptr;
        v->baked_alloc_res = 0;
        CU(mrp::dev_malloc(&v->baked, (size_t)B * B * B * sizeof(float)));
        v->baked_alloc_res = B;
    }
    v->bk_res = B;
    VolumeDev d = v->dev();
    CU(launch_baked_tr(v->baked, d, B, alpha, L, v->params.seed, v->params.bake_replicate_seeding, g.sms, v->stream));
    v->baked_gtex_ok = false;
    v->has_baked = true;
    v->bk_alpha = alpha;
    v->bk_seed = v->params.seed;
    std::memcpy(v->bk_light, L, sizeof v->bk_light);
    return MRP_OK;
}

}  // namespace mrpi
extern "C" {

mrp_status mrp_update_hg_lut(mrp_volume* v, float g_) {
    TRY(need_init());
    if (!v) return fail(MRP_ERR_INVALID, "null volume");
    TRY(update_lut_async(v, g_));
    CU(cudaStreamSynchronize(v->stream));
    return MRP_OK;
}
mrp_status mrp_update_tr(mrp_volume* v, const float light_dir[3], float alpha) {
    TRY(need_init());
    if (!v || !light_dir) return fail(MRP_ERR_INVALID, "null argument");
    TRY(update_tr_async(v, light_dir, alpha));
    CU(cudaStreamSynchronize(v->stream));
    return MRP_OK;
}
mrp_status mrp_update_baked_tr(mrp_volume* v, const float light_dir[3], float alpha) {
    TRY(need_init());
    if (!v || !light_dir) return fail(MRP_ERR_INVALID, "null argument");
    if (!v->has_data) return fail(MRP_ERR_NOT_READY, "no data");
    TRY(update_baked_async(v, light_dir, alpha));
    CU(cudaStreamSynchronize(v->stream));
    return MRP_OK;
}

// --- rendering ----------------------------------------------------------------
}  // extern "C"
namespace mrpi {
mrp_status ensure_predictor_buffers(mrp_volume* v, size_t npix) {
    if (v->rec_cap >= npix) return MRP_OK;
    mrp::dev_free(v->rec_count); mrp::dev_free(v->rec_pix); mrp::dev_free(v->rec_f); mrp::dev_free(v->feat);
    v->rec_count = nullptr; v->rec_pix = nullptr; v->rec_f = nullptr; v->feat = nullptr; v->rec_cap = 0;
    CU(mrp::dev_malloc(&v->rec_count, 2 * sizeof(int)));   // records, the march's pixel chunks
    CU(mrp::dev_malloc(&v->rec_pix, npix * sizeof(int)));
    CU(mrp::dev_malloc(&v->rec_f, npix * 16 * sizeof(float)));
    CU(mrp::dev_malloc(&v->feat, tiled_feature_floats(npix) * sizeof(float)));
    CU(tc_ensure_scratch(v->tc));
    v->rec_cap = npix;
    return MRP_OK;
}
mrp_status ensure_accum(mrp_volume* v, size_t npix) {
    if (v->accum_pix >= npix) return MRP_OK;
    mrp::dev_free(v->accum);
    v->accum = nullptr;
    v->accum_pix = 0;
    CU(mrp::dev_malloc(&v->accum, npix * sizeof(float4)));
    v->accum_pix = npix;
    return MRP_OK;
}
}  // namespace mrpi
extern "C" {

}  // extern "C"
namespace mrpi {
ViewDev make_view(const mrp_volume* v, const mrp_view* w, int frame, int mean_k) {
    ViewDev d{};
    d.width = w->width;
    d.height = w->height;
    d.ori = {w->ori[0], w->ori[1], w->ori[2]};
    d.up = {w->up[0], w->up[1], w->up[2]};
    d.right = {w->right[0], w->right[1], w->right[2]};
    d.light_dir = {w->light_dir[0], w->light_dir[1], w->light_dir[2]};
    d.light_color = {w->light_color[0], w->light_color[1], w->light_color[2]};
    d.alpha = w->alpha;
    d.g = w->g;
    d.multi_scatter = w->multi_scatter;
    d.spp = w->spp;
    d.seed = w->seed;
    d.frame = frame;
    d.mean_k = mean_k;
    float t_step = 2.0f / (float)v->res;
    float smax = v->max_density * w->alpha;
    d.pass_rate = std::exp(-t_step * smax);
    return d;
}
}  // namespace mrpi
extern "C" {

static mrp_status render_impl(mrp_volume* v, const mrp_view* w, mrp_render_type type, int sample_num, float* out,
                              int out_is_device, unsigned long long* counters, bool async = false);

mrp_status mrp_render(mrp_volume* v, const mrp_view* w, mrp_render_type type, int sample_num, float* out, int out_is_device) {
    return render_impl(v, w, type, sample_num, out, out_is_device, nullptr);
}

mrp_status mrp_render_start(mrp_volume* v, const mrp_view* w, mrp_render_type type, int sample_num, float* out,
                            int out_is_device) {
    return render_impl(v, w, type, sample_num, out, out_is_device, nullptr, true);
}

mrp_status mrp_render_wait(mrp_volume* v, int keep) {
    TRY(need_init());
    if (!v) return fail(MRP_ERR_INVALID, "null volume");
    if (keep != 0 && keep != 1) return fail(MRP_ERR_INVALID, "keep must be 0 or 1");
    if (keep == 1) {
        // every result but the newest: the second newest start used the slot
        // the next start will take, and its copy event has not been re-recorded
        if (v->async_inflight >= 2) CU(cudaEventSynchronize(v->ev_copied[v->async_slot]));
        if (v->async_inflight > 1) v->async_inflight = 1;
        return MRP_OK;
    }
    CU(cudaStreamSynchronize(v->stream));
    CU(cudaStreamSynchronize(v->stream_copy));
    v->async_inflight = 0;
    if (v->async_tc) {   // the error flag gathers every tensor-core launch since the last wait
        v->async_tc = false;
        int herr = 0;
        CU(cudaMemcpy(&herr, v->tc.d + 1, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) return fail(MRP_ERR_TIMEOUT, "tensor-core MLP: MMA completion wait timed out");
    }
    return MRP_OK;
}

mrp_status mrp_render_counters(mrp_volume* v, const mrp_view* w, mrp_render_type type, unsigned long long counters[4]) {
    TRY(need_init());
    if (!counters) return fail(MRP_ERR_INVALID, "null argument");
    unsigned long long* d = nullptr;
    CU(mrp::dev_malloc(&d, 4 * sizeof(unsigned long long)));
    cudaMemset(d, 0, 4 * sizeof(unsigned long long));
    float* out = nullptr;
    size_t npix = (size_t)std::max(w ? w->width : 0, 0) * std::max(w ? w->height : 0, 0);
    if (mrp::dev_malloc(&out, std::max<size_t>(npix, 1) * 16) != cudaSuccess) { mrp::dev_free(d); return fail(MRP_ERR_OOM, "counters"); }
    mrp_status st = render_impl(v, w, type, 1, out, 1, d);
    if (st == MRP_OK && cudaMemcpy(counters, d, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
        st = fail(MRP_ERR_CUDA, "counters readback");
    mrp::dev_free(d);
    mrp::dev_free(out);
    return st;
}

static mrp_status render_impl(mrp_volume* v, const mrp_view* w, mrp_render_type type, int sample_num, float* out,
                              int out_is_device, unsigned long long* counters, bool async) {
    TRY(need_init());
    // a synchronous render (or counter run) first lets started ones finish
    if (v && !async && v->async_inflight) TRY(mrp_render_wait(v, 0));
    if (!v || !w || !out) return fail(MRP_ERR_INVALID, "null argument");
    if (w->width <= 0 || w->height <= 0 || (long long)w->width * w->height > (1ll << 28))
        return fail(MRP_ERR_INVALID, "image size %dx%d", w->width, w->height);
    if (sample_num < 1) return fail(MRP_ERR_INVALID, "sample_num must be >= 1");
    if (type == MRP_RPNN) return fail(MRP_ERR_UNSUPPORTED, "RPNN is compiled only with -DCRPNN in the reference");
    if (type != MRP_PT && type != MRP_MRPNN) return fail(MRP_ERR_INVALID, "unknown render type %d", (int)type);
    if (!v->has_data) return fail(MRP_ERR_NOT_READY, "no volume data");
    if (type == MRP_MRPNN && !v->has_pyramid) return fail(MRP_ERR_NOT_READY, "MRPNN needs the pyramid (mrp_volume_update)");
    if (type == MRP_PT && (w->spp < 1 || w->multi_scatter < 1)) return fail(MRP_ERR_INVALID, "PT needs spp, multi_scatter >= 1");
    size_t npix = (size_t)w->width * w->height;
    // buffers that must grow are freed and reallocated: not under copies in flight
    if (v->async_inflight && (v->accum_pix < npix || v->accum_alt_pix < npix || (type == MRP_PT && v->trace_pix < npix) ||
                              (type == MRP_MRPNN && v->rec_cap < npix)))
        TRY(mrp_render_wait(v, 0));
    TRY(ensure_accum(v, npix));
    if (type == MRP_PT && v->trace_pix < npix) {
        mrp::dev_free(v->sum3); mrp::dev_free(v->first_pos); mrp::dev_free(v->counter);
        v->sum3 = nullptr; v->first_pos = nullptr; v->counter = nullptr; v->trace_pix = 0;
        CU(mrp::dev_malloc(&v->sum3, npix * 3 * sizeof(double)));
        CU(mrp::dev_malloc(&v->first_pos, npix * sizeof(int)));
        CU(mrp::dev_malloc(&v->counter, sizeof(unsigned long long)));
        v->trace_pix = npix;
    }
    // caches first (the reference updates them inside its launch loop,
    // core/volume.cu:511-518; they do not change between its launches)
    // with an environment map each predictor launch picks its light from the
    // map or the sun (core/volume.cu:494-509) and updates the TR levels for it
    const bool env_light = type == MRP_MRPNN && v->hdri;
    if (type == MRP_MRPNN) {
        TRY(update_lut_async(v, w->g));
        if (!env_light) TRY(update_tr_async(v, w->light_dir, w->alpha));
    } else if (v->params.nee_mode == 0) {
        TRY(update_baked_async(v, w->light_dir, w->alpha));
    }
    if (type == MRP_MRPNN) TRY(ensure_predictor_buffers(v, npix));
    // result buffer: accum, or for a started render the slot's own buffer,
    // reused only after the copy out of its previous result is done
    const int slot = async ? v->async_slot : 0;
    if (slot == 1 && v->accum_alt_pix < npix) {
        mrp::dev_free(v->accum_alt);
        v->accum_alt = nullptr;
        v->accum_alt_pix = 0;
        CU(mrp::dev_malloc(&v->accum_alt, npix * sizeof(float4)));
        v->accum_alt_pix = npix;
    }
    float4* const acc = slot == 1 ? v->accum_alt : v->accum;
    if (async) CU(cudaStreamWaitEvent(v->stream, v->ev_copied[slot], 0));
    VolumeDev d = v->dev();
    const bool tc_net = type == MRP_MRPNN && v->params.precision != MRP_FP32;
    if (tc_net && !(async && v->async_tc)) CU(cudaMemsetAsync(v->tc.d + 1, 0, sizeof(int), v->stream));
    CU(cudaEventRecord(v->ev0, v->stream));
    for (int i = 0; i < sample_num; ++i) {
        mrp_view wi = *w;
        if (env_light) {
            env_light_for_launch(v, (uint32_t)(w->frame_offset + i), w->seed, wi.light_dir, wi.light_color);
            TRY(update_tr_async(v, wi.light_dir, wi.alpha));
        }
        ViewDev vd = make_view(v, &wi, w->frame_offset + i, i);
        vd.counters = counters;
        bool last = i == sample_num - 1;
        if (type == MRP_MRPNN) {
            HitRecords rec = v->records();
            if (last) CU(cudaEventRecord(v->ev0, v->stream));
            CU(launch_hit(d, vd, rec, acc, v->stream));
            if (last) CU(cudaEventRecord(v->ev_stage[0], v->stream));
            CU(launch_gather_rec(d, vd, rec, v->feat, v->params.precision != MRP_FP32, v->stream));
            if (last) CU(cudaEventRecord(v->ev_stage[1], v->stream));
            if (v->params.precision == MRP_FP32) {
                CU(launch_mlp_rec_fp32(d, vd, rec, v->feat, g.d_weights, acc, v->stream));
            } else {
                CU(tc_launch_mlp_rec(g.tc, v->params.precision == MRP_FP8, d, vd, rec, v->feat, acc, v->tc, g.sms,
                                     v->stream));
            }
        } else {
            CU(cudaMemsetAsync(v->sum3, 0, npix * 3 * sizeof(double), v->stream));
            CU(launch_fill_int(v->first_pos, (int)npix, w->spp, v->stream));
            CU(cudaMemsetAsync(v->counter, 0, sizeof(unsigned long long), v->stream));
            if (last) CU(cudaEventRecord(v->ev0, v->stream));
            VolumeDev dt = d;
            if (v->params.tracer_filter) {
                TRY(ensure_density_texture(v));
                dt.dens_tex = v->dens_tex;
                if (v->params.nee_mode == 0) {
                    TRY(ensure_baked_texture(v));
                    dt.baked_tex = v->baked_gtex.tex;
                }
            }
            CU(launch_trace(dt, vd, v->sum3, nullptr, v->first_pos, v->counter, g.sms, v->stream));
            if (last) CU(cudaEventRecord(v->ev_stage[0], v->stream));
            CU(launch_trace_resolve(v->sum3, v->first_pos, (int)npix, w->spp, i, acc, v->stream));
            if (last) CU(cudaEventRecord(v->ev_stage[1], v->stream));
        }
    }
    CU(cudaEventRecord(v->ev1, v->stream));
    if (async) {
        // the copy out runs on stream_copy beside the next render's kernels
        CU(cudaEventRecord(v->ev_done[slot], v->stream));
        CU(cudaStreamWaitEvent(v->stream_copy, v->ev_done[slot], 0));
        CU(cudaMemcpyAsync(out, acc, npix * sizeof(float4), out_is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           v->stream_copy));
        CU(cudaEventRecord(v->ev_copied[slot], v->stream_copy));
        v->async_slot ^= 1;
        v->async_inflight++;
        v->async_tc = v->async_tc || tc_net;
        v->stages_valid = false;
        return MRP_OK;
    }
    CU(cudaMemcpyAsync(out, acc, npix * sizeof(float4), out_is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       v->stream));
    CU(cudaStreamSynchronize(v->stream));
    if (sample_num == 1) CU(cudaEventElapsedTime(&v->last_ms, v->ev0, v->ev1));
    else v->last_ms = -1.0f;
    CU(cudaEventElapsedTime(&v->stage_ms[0], v->ev0, v->ev_stage[0]));
    CU(cudaEventElapsedTime(&v->stage_ms[1], v->ev_stage[0], v->ev_stage[1]));
    CU(cudaEventElapsedTime(&v->stage_ms[2], v->ev_stage[1], v->ev1));
    v->stages_valid = true;
    if (type == MRP_MRPNN && v->params.precision != MRP_FP32) {
        int herr = 0;
        CU(cudaMemcpy(&herr, v->tc.d + 1, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) return fail(MRP_ERR_TIMEOUT, "tensor-core MLP: MMA completion wait timed out");
    }
    return MRP_OK;
}

mrp_status mrp_last_render_stages(const mrp_volume* v, float ms[3]) {
    if (!v || !ms) return fail(MRP_ERR_INVALID, "null argument");
    if (!v->stages_valid) return fail(MRP_ERR_NOT_READY, "no render yet");
    for (int i = 0; i < 3; ++i) ms[i] = v->stage_ms[i];
    return MRP_OK;
}

mrp_status mrp_render_predict_debug(mrp_volume* v, const mrp_view* w, float* rgba, float* aux, float* feat,
                                    int is_device) {
    TRY(need_init());
    if (!v || !w || !rgba || !aux || !feat) return fail(MRP_ERR_INVALID, "null argument");
    if (w->width <= 0 || w->height <= 0 || (long long)w->width * w->height > (1ll << 22))
        return fail(MRP_ERR_INVALID, "debug render limited to 4M pixels");
    if (!v->has_pyramid) return fail(MRP_ERR_NOT_READY, "MRPNN needs the pyramid (mrp_volume_update)");
    size_t npix = (size_t)w->width * w->height;
    TRY(update_lut_async(v, w->g));
    TRY(update_tr_async(v, w->light_dir, w->alpha));
    float4* acc = nullptr;
    float *da = aux, *df = feat;
    std::vector<void*> allocs;
    auto alloc = [&](size_t b) { void* p = nullptr; if (mrp::dev_malloc(&p, b) == cudaSuccess) allocs.push_back(p); return p; };
    auto release = [&]() { for (void* p : allocs) mrp::dev_free(p); };
    acc = (float4*)alloc(npix * sizeof(float4));
    if (!is_device) { da = (float*)alloc(npix * 20 * 4); df = (float*)alloc(npix * 576 * 4); }
    if (!acc || !da || !df) { release(); return fail(MRP_ERR_OOM, "debug render buffers"); }
    cudaMemsetAsync(df, 0, npix * 576 * 4, v->stream);
    cudaMemsetAsync(da, 0, npix * 20 * 4, v->stream);
    ViewDev vd = make_view(v, w, w->frame_offset, 0);
    mrp_status ps = ensure_predictor_buffers(v, npix);
    if (ps != MRP_OK) { release(); return ps; }
    HitRecords rec = v->records();
    VolumeDev dv = v->dev();
    // the volume's precision: fp32 features and the FP32 network, or the
    // fp16 features and the tensor-core network of mrp_render
    const bool tc = v->params.precision != MRP_FP32;
    cudaError_t e = tc ? tc_ensure_scratch(v->tc) : cudaSuccess;
    if (e == cudaSuccess && tc) e = cudaMemsetAsync(v->tc.d + 1, 0, sizeof(int), v->stream);
    if (e == cudaSuccess) e = launch_hit(dv, vd, rec, acc, v->stream);
    if (e == cudaSuccess) e = launch_gather_rec(dv, vd, rec, v->feat, tc, v->stream);
    if (e == cudaSuccess) {
        e = tc ? tc_launch_mlp_rec(g.tc, v->params.precision == MRP_FP8, dv, vd, rec, v->feat, acc, v->tc, g.sms,
                                   v->stream)
               : launch_mlp_rec_fp32(dv, vd, rec, v->feat, g.d_weights, acc, v->stream);
    }
    if (e == cudaSuccess) e = launch_debug_scatter(rec, v->feat, tc, (int)npix, da, df, v->stream);
    cudaMemcpyKind k = is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (e == cudaSuccess) {
        cudaMemcpyAsync(rgba, acc, npix * sizeof(float4), k, v->stream);
        if (!is_device) {
            cudaMemcpyAsync(aux, da, npix * 20 * 4, k, v->stream);
            cudaMemcpyAsync(feat, df, npix * 576 * 4, k, v->stream);
        }
    }
    cudaError_t e2 = cudaStreamSynchronize(v->stream);
    release();
    if (e != cudaSuccess || e2 != cudaSuccess)
        return fail(MRP_ERR_CUDA, "debug render: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    if (tc) {
        int herr = 0;
        CU(cudaMemcpy(&herr, v->tc.d + 1, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) return fail(MRP_ERR_TIMEOUT, "tensor-core MLP: MMA completion wait timed out");
    }
    return MRP_OK;
}

mrp_status mrp_tc_gemm_check(int fp8, const float* A, const float* B, int n, int k, float* D) {
    TRY(need_init());
    if (!A || !B || !D || n < 16 || n > 128 || n % 16 || k < 16 || k > 128 || k % (fp8 ? 32 : 16))
        return fail(MRP_ERR_INVALID, "tc gemm check: n in 16..128 step 16, k multiple of %d up to 128", fp8 ? 32 : 16);
    std::lock_guard<std::mutex> lk(g.mu);
    size_t bytes = (size_t)(128 * k + n * k + 128 * n) * sizeof(float) + 64;
    TRY(ensure_scratch(bytes));
    float* dA = (float*)g.scratch;
    float* dB = dA + 128 * k;
    float* dD = dB + n * k;
    int* derr = (int*)(dD + 128 * n);
    CU(cudaMemcpyAsync(dA, A, 128 * k * sizeof(float), cudaMemcpyHostToDevice, g.stream));
    CU(cudaMemcpyAsync(dB, B, (size_t)n * k * sizeof(float), cudaMemcpyHostToDevice, g.stream));
    CU(cudaMemsetAsync(derr, 0, sizeof(int), g.stream));
    CU(tc_gemm_test(fp8 != 0, dA, dB, n, k, dD, derr, g.stream));
    int herr = 0;
    CU(cudaMemcpyAsync(D, dD, (size_t)128 * n * sizeof(float), cudaMemcpyDeviceToHost, g.stream));
    CU(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, g.stream));
    CU(cudaStreamSynchronize(g.stream));
    if (herr) return fail(MRP_ERR_TIMEOUT, "tensor-core GEMM check: MMA completion wait timed out");
    return MRP_OK;
}

mrp_status mrp_last_render_ms(const mrp_volume* v, float* ms) {
    if (!v || !ms) return fail(MRP_ERR_INVALID, "null argument");
    *ms = v->last_ms;
    return MRP_OK;
}

// --- parity entry points --------------------------------------------------------
mrp_status mrp_predict_features(const float* feat, const float* gamma, float g_, const float sr[3], int n, float* out3,
                                mrp_precision precision, int is_device) {
    TRY(need_init());
    if (!feat || !gamma || !sr || !out3 || n < 0) return fail(MRP_ERR_INVALID, "null argument");
    if (n == 0) return MRP_OK;
    std::lock_guard<std::mutex> lk(g.mu);
    const float *df = feat, *dg = gamma;
    float* dout = out3;
    if (!is_device) {
        size_t need = (size_t)n * (576 + 1 + 3) * sizeof(float);
        TRY(ensure_scratch(need));
        float* base = (float*)g.scratch;
        float* f = base;
        float* gm = base + (size_t)n * 576;
        dout = gm + n;
        CU(cudaMemcpyAsync(f, feat, (size_t)n * 576 * sizeof(float), cudaMemcpyHostToDevice, g.stream));
        CU(cudaMemcpyAsync(gm, gamma, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, g.stream));
        df = f;
        dg = gm;
    }
    if (precision == MRP_FP32) {
        CU(launch_mlp_fp32(g.d_weights, df, dg, g_, sr, n, dout, g.stream));
    } else if (precision == MRP_BF16 || precision == MRP_FP8) {
        CU(cudaMemsetAsync(g.tc.d_err, 0, sizeof(int), g.stream));
        CU(tc_launch_mlp(g.tc, precision == MRP_FP8, df, dg, g_, sr, n, dout, g.sms, g.stream));
        int herr = 0;
        CU(cudaMemcpyAsync(&herr, g.tc.d_err, sizeof(int), cudaMemcpyDeviceToHost, g.stream));
        CU(cudaStreamSynchronize(g.stream));
        if (herr) return fail(MRP_ERR_TIMEOUT, "tensor-core MLP: MMA completion wait timed out");
    } else {
        return fail(MRP_ERR_INVALID, "unknown precision %d", (int)precision);
    }
    if (!is_device) CU(cudaMemcpyAsync(out3, dout, (size_t)n * 3 * sizeof(float), cudaMemcpyDeviceToHost, g.stream));
    CU(cudaStreamSynchronize(g.stream));
    return MRP_OK;
}

}  // extern "C"

// --- mrp_predict_features_noalloc ----------------------------------------------------
// One fixed scratch array per device, part of this library's device image.
// Host code must not hand `g_noalloc_scratch` itself to a kernel: on the host
// that name is only a stand-in for the device symbol.  Its device address is
// looked up once per device (cudaGetSymbolAddress, with the device current)
// and passed on.  Layout, every part on a 256-byte boundary:
//   [0, 4)     tile counter of the tensor-core network  (zeroed before each launch)
//   [4, 8)     error flag of the tensor-core network    (zeroed before each launch)
//   [256, ..)  feat  [MRP_NOALLOC_MAX_POINTS][576] fp32 (copied in; no clearing)
//   then       gamma [MRP_NOALLOC_MAX_POINTS] fp32
//   then       out   [MRP_NOALLOC_MAX_POINTS][3] fp32
static __device__ __align__(256) unsigned char g_noalloc_scratch[MRP_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr size_t kNoAllocFeat = 256;
constexpr size_t kNoAllocGamma = kNoAllocFeat + (size_t)MRP_NOALLOC_MAX_POINTS * 576 * sizeof(float);
constexpr size_t kNoAllocOut = kNoAllocGamma + (size_t)MRP_NOALLOC_MAX_POINTS * sizeof(float);
static_assert(kNoAllocOut + (size_t)MRP_NOALLOC_MAX_POINTS * 3 * sizeof(float) == MRP_NOALLOC_SCRATCH_BYTES,
              "scratch layout");
static_assert(kNoAllocGamma % 256 == 0 && kNoAllocOut % 256 == 0, "scratch alignment");
constexpr int kNoAllocDevices = 64;
unsigned char* g_noalloc_addr[kNoAllocDevices] = {};   // device address per device, set under g.mu

// Makes `dev` current for the scope and restores the caller's device after.
struct CurrentDevice {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit CurrentDevice(int dev) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != dev) err = cudaSetDevice(dev);
    }
    ~CurrentDevice() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};
}  // namespace

extern "C" {

mrp_status mrp_predict_features_noalloc(const float* feat, const float* gamma, float g_, const float sr[3], int n,
                                        float* out3, mrp_precision precision) {
    TRY(need_init());
    if (!feat || !gamma || !sr || !out3 || n < 0) return fail(MRP_ERR_INVALID, "null argument");
    if (n > MRP_NOALLOC_MAX_POINTS)
        return fail(MRP_ERR_INVALID,
                    "mrp_predict_features_noalloc: %d points exceed its fixed scratch of %d points; split the batch",
                    n, MRP_NOALLOC_MAX_POINTS);
    if (precision != MRP_FP32 && precision != MRP_BF16 && precision != MRP_FP8)
        return fail(MRP_ERR_INVALID, "unknown precision %d", (int)precision);
    if (n == 0) return MRP_OK;
    std::lock_guard<std::mutex> lk(g.mu);
    if (g.device < 0 || g.device >= kNoAllocDevices) return fail(MRP_ERR_INVALID, "device %d", g.device);
    CurrentDevice cd(g.device);
    CU(cd.err);
    unsigned char*& base = g_noalloc_addr[g.device];
    if (!base) CU(cudaGetSymbolAddress((void**)&base, g_noalloc_scratch));
    int* counter = (int*)base;
    int* err = (int*)(base + 4);
    float* f = (float*)(base + kNoAllocFeat);
    float* gm = (float*)(base + kNoAllocGamma);
    float* dout = (float*)(base + kNoAllocOut);
    CU(cudaMemcpyAsync(f, feat, (size_t)n * 576 * sizeof(float), cudaMemcpyHostToDevice, g.stream));
    CU(cudaMemcpyAsync(gm, gamma, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, g.stream));
    int herr = 0;
    if (precision == MRP_FP32) {
        CU(launch_mlp_fp32(g.d_weights, f, gm, g_, sr, n, dout, g.stream));
    } else {
        CU(tc_launch_mlp_at(g.tc, precision == MRP_FP8, f, gm, g_, sr, n, dout, counter, err, g.sms, g.stream));
        CU(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, g.stream));
    }
    CU(cudaMemcpyAsync(out3, dout, (size_t)n * 3 * sizeof(float), cudaMemcpyDeviceToHost, g.stream));
    CU(cudaStreamSynchronize(g.stream));
    if (herr) return fail(MRP_ERR_TIMEOUT, "tensor-core MLP: MMA completion wait timed out");
    return MRP_OK;
}

mrp_status mrp_gather_features(mrp_volume* v, const float* pos, const float* bases, const float L[3], float g_, float alpha,
                               int n, float* feat, float* gamma, int is_device) {
    TRY(need_init());
    if (!v || !pos || !bases || !L || !feat || !gamma || n < 0) return fail(MRP_ERR_INVALID, "null argument");
    if (!v->has_pyramid || !v->has_tr || !v->has_lut) return fail(MRP_ERR_NOT_READY, "gather needs pyramid, TR mips and LUT");
    if (n == 0) return MRP_OK;
    float* dl = nullptr;
    float *dp = (float*)pos, *db = (float*)bases, *dfeat = feat, *dgam = gamma;
    std::vector<void*> allocs;
    auto alloc = [&](size_t bytes) -> float* { void* p = nullptr; if (mrp::dev_malloc(&p, bytes) != cudaSuccess) return nullptr; allocs.push_back(p); return (float*)p; };
    auto release = [&]() { for (void* p : allocs) mrp::dev_free(p); };
    dl = alloc(3 * sizeof(float));
    if (!dl) { release(); return fail(MRP_ERR_OOM, "gather scratch"); }
    cudaMemcpyAsync(dl, L, 3 * sizeof(float), cudaMemcpyHostToDevice, v->stream);
    if (!is_device) {
        dp = alloc((size_t)n * 3 * 4); db = alloc((size_t)n * 12 * 4); dfeat = alloc((size_t)n * 576 * 4); dgam = alloc((size_t)n * 4);
        if (!dp || !db || !dfeat || !dgam) { release(); return fail(MRP_ERR_OOM, "gather scratch"); }
        cudaMemcpyAsync(dp, pos, (size_t)n * 3 * 4, cudaMemcpyHostToDevice, v->stream);
        cudaMemcpyAsync(db, bases, (size_t)n * 12 * 4, cudaMemcpyHostToDevice, v->stream);
    }
    cudaError_t e = launch_gather(v->dev(), dp, db, dl, g_, alpha, n, dfeat, dgam, v->stream);
    if (e == cudaSuccess && !is_device) {
        cudaMemcpyAsync(feat, dfeat, (size_t)n * 576 * 4, cudaMemcpyDeviceToHost, v->stream);
        cudaMemcpyAsync(gamma, dgam, (size_t)n * 4, cudaMemcpyDeviceToHost, v->stream);
    }
    cudaError_t e2 = cudaStreamSynchronize(v->stream);
    release();
    if (e != cudaSuccess || e2 != cudaSuccess)
        return fail(MRP_ERR_CUDA, "gather: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    return MRP_OK;
}

mrp_status mrp_first_hit(mrp_volume* v, const float* ori, const float* dir, float alpha, int n, float* hit4, int is_device) {
    TRY(need_init());
    if (!v || !ori || !dir || !hit4 || n < 0) return fail(MRP_ERR_INVALID, "null argument");
    if (!v->has_data) return fail(MRP_ERR_NOT_READY, "no data");
    if (n == 0) return MRP_OK;
    float pass_rate = std::exp(-(2.0f / (float)v->res) * (v->max_density * alpha));
    const float *dori = ori, *ddir = dir;
    float* dhit = hit4;
    float* tmp = nullptr;
    if (!is_device) {
        CU(mrp::dev_malloc(&tmp, (size_t)n * 10 * sizeof(float)));
        float* o = tmp; float* d = tmp + 3 * (size_t)n; dhit = tmp + 6 * (size_t)n;
        cudaMemcpyAsync(o, ori, (size_t)n * 12, cudaMemcpyHostToDevice, v->stream);
        cudaMemcpyAsync(d, dir, (size_t)n * 12, cudaMemcpyHostToDevice, v->stream);
        dori = o; ddir = d;
    }
    cudaError_t e = launch_first_hit(v->dev(), dori, ddir, alpha, pass_rate, n, dhit, v->stream);
    if (e == cudaSuccess && !is_device) cudaMemcpyAsync(hit4, dhit, (size_t)n * 16, cudaMemcpyDeviceToHost, v->stream);
    cudaError_t e2 = cudaStreamSynchronize(v->stream);
    if (tmp) mrp::dev_free(tmp);
    if (e != cudaSuccess || e2 != cudaSuccess) return fail(MRP_ERR_CUDA, "first_hit: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    return MRP_OK;
}

}  // extern "C"
