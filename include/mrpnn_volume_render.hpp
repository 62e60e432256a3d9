// mrpnn_volume_render.hpp -- the reference's VolumeRender and Camera classes
// (core/volume.hpp:45-155, core/camera.hpp:29-43) rebuilt over the C ABI of
// libmrpnn_b200.so (include/mrpnn.h), header-only.
//
// Drop-in: same class and method names, argument order and defaults for the
// render path (SetData/SetDatas -> Update -> Render, Camera::RenderToFile).
// Differences, all from the C ABI: errors throw mrpnn::Error instead of being
// printed and ignored (core/volume.cu:15); max_density is computed by Update
// (the reference leaves 1e-5 for user data); SkyBox is a constant radiance
// (SetSky) instead of an HDRI; the interactive Render overload and
// GatherData are not part of this path.
//
// Build: g++ -std=c++17 -I<repo>/include -I/usr/local/cuda/include app.cpp
//        -L<repo>/mrpnn_b200 -lmrpnn_b200 -Wl,-rpath,<repo>/mrpnn_b200
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include <vector_types.h>   // float3, float4, int2 (CUDA toolkit, header only)

#include "mrpnn.h"

namespace mrpnn {

struct Error : std::runtime_error {
    mrp_status status;
    Error(mrp_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};
inline void check(mrp_status s, const char* where) {
    if (s != MRP_OK) throw Error(s, std::string(where) + ": " + mrp_last_error());
}
inline void ensure_init(int device = 0) {
    static bool done = false;
    if (!done) {
        check(mrp_init(device, nullptr), "mrp_init");
        done = true;
    }
}

}  // namespace mrpnn

typedef std::function<float(int x, int y, int z, float u, float v, float w)> FillFunc;

class VolumeRender {
   public:
    enum RenderType { PT, RPNN, MRPNN };   // core/volume.hpp:98-100

    float max_density = 0.00001f;           // refreshed by Update()
    float min_val = 0.0f;

    explicit VolumeRender(int resolution) : resolution(resolution) {
        mrpnn::ensure_init();
        mrpnn::check(mrp_volume_create(resolution, &h), "VolumeRender");
        mrp_default_params(&params);
        datas.assign((size_t)resolution * resolution * resolution, 0.0f);
    }
    // The same with the device grid in fp16 (MRP_STORAGE_FP16): half the
    // HBM; the host copy `datas` stays float, as the reference's.
    VolumeRender(int resolution, mrp_storage storage) : resolution(resolution) {
        mrpnn::ensure_init();
        mrpnn::check(mrp_volume_create_ex(resolution, storage, &h), "VolumeRender");
        mrp_default_params(&params);
        datas.assign((size_t)resolution * resolution * resolution, 0.0f);
    }
    // VolumeRender(string path, bool cacheTR) -> LoadData (core/volume.cu:959-1149):
    // .bin / .txt / .vox (and the .bin cache beside a parsed file); Update
    // has run.  cacheTR has no effect: the baked TR grid is sized by
    // SetBakeResolution, not by the load.
    explicit VolumeRender(const std::string& path, bool /*cacheTR*/ = false) {
        mrpnn::ensure_init();
        mrpnn::check(mrp_volume_file_read(path.c_str(), &resolution, nullptr, 0), "VolumeRender(path)");
        datas.assign((size_t)resolution * resolution * resolution, 0.0f);
        mrpnn::check(mrp_volume_file_read(path.c_str(), &resolution, datas.data(), datas.size()), "VolumeRender(path)");
        mrpnn::check(mrp_volume_load(path.c_str(), 1, &h), "VolumeRender(path)");
        mrp_default_params(&params);
        mrp_volume_info info;
        mrpnn::check(mrp_volume_get_info(h, &info), "VolumeRender(path)");
        max_density = info.max_density;
        dirty = false;
    }
    ~VolumeRender() { mrp_volume_destroy(h); }
    VolumeRender(const VolumeRender&) = delete;
    VolumeRender& operator=(const VolumeRender&) = delete;

    // core/volume.cu:1178-1184
    void SetData(int x, int y, int z, float value) {
        datas[((size_t)x * resolution + y) * resolution + z] = value;
        dirty = true;
    }
    // ParallelFill semantics (core/omp.cpp:4-18): u = (x + 0.5) / resolution
    void SetDatas(FillFunc func) {
        int R = resolution;
        unsigned nt = std::max(1u, std::thread::hardware_concurrency());
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                for (int i = (int)t; i < R; i += (int)nt)
                    for (int j = 0; j < R; ++j)
                        for (int k = 0; k < R; ++k) {
                            float u = (float)((i + 0.5) / R), v = (float)((j + 0.5) / R), w = (float)((k + 0.5) / R);
                            datas[((size_t)i * R + j) * R + k] = func(i, j, k, u, v, w);
                        }
            });
        for (auto& t : th) t.join();
        dirty = true;
    }
    // core/volume.cu:1443-1531
    void Update(bool process_mips = true, bool need_reset_datas_dev = true) {
        if (dirty || need_reset_datas_dev) {
            mrpnn::check(mrp_volume_set_data(h, datas.data(), resolution, 0), "SetData");
            dirty = false;
        }
        mrpnn::check(mrp_volume_update(h, process_mips ? 1 : 0), "Update");
        mrp_volume_info info;
        mrpnn::check(mrp_volume_get_info(h, &info), "Update");
        max_density = info.max_density;
    }
    void Update_TR(float3 lightDir, float alpha = 64.0f, bool /*CPU*/ = false) {
        float L[3] = {lightDir.x, lightDir.y, lightDir.z};
        mrpnn::check(mrp_update_tr(h, L, alpha), "Update_TR");
    }
    void UpdateHGLut(float g) { mrpnn::check(mrp_update_hg_lut(h, g), "UpdateHGLut"); }
    // core/volume.cu:1424-1442, on a host copy of the current table (read
    // back once per table)
    float GetHGLut(float cos, float angle) {
        mrp_volume_info info;
        mrpnn::check(mrp_volume_get_info(h, &info), "GetHGLut");
        if (!info.has_lut) throw std::runtime_error("GetHGLut: no HG table yet (UpdateHGLut)");
        if (lut_host.empty() || lut_host_g != info.lut_g) {
            size_t n = 0;
            mrpnn::check(mrp_volume_read(h, MRP_RES_LUT, 0, nullptr, &n, 0), "GetHGLut");
            lut_host.assign(n, 0.0f);
            mrpnn::check(mrp_volume_read(h, MRP_RES_LUT, 0, lut_host.data(), &n, 0), "GetHGLut");
            lut_host_g = info.lut_g;
        }
        float r = 0.0f;
        mrpnn::check(mrp_hg_lut_lookup(lut_host.data(), cos, angle, &r), "GetHGLut");
        return r;
    }

    void SetScatterRate(float rate) { SetScatterRate(float3{rate, rate, rate}); }
    void SetScatterRate(float3 rate) {
        params.scatter_rate[0] = rate.x; params.scatter_rate[1] = rate.y; params.scatter_rate[2] = rate.z;
        push();
    }
    void SetTrScale(float scale) { params.tr_scale = scale; push(); }
    void SetEnvExp(float exp) { params.env_exp = exp; push(); }
    void SetExposure(float exp) { exposure = exp; }          // interactive tone mapping only
    void SetCheckboard(bool checkboard) { this->checkboard = checkboard; }
    void SetSurfaceIOR(float ior) { this->ior = ior; }       // marching mode only
    // core/volume.cu:1696-1728: a Radiance .hdr file as the environment map
    void SetHDRI(const std::string& path) { mrpnn::check(mrp_volume_load_hdri(h, path.c_str()), "SetHDRI"); }
    // Constant environment radiance, used while no map is set.
    void SetSky(float3 radiance) {
        params.sky[0] = radiance.x; params.sky[1] = radiance.y; params.sky[2] = radiance.z;
        push();
    }
    void SetPrecision(mrp_precision p) { params.precision = p; push(); }
    // texture-unit filtering (the reference's tex3D / tex2D) for the tracer's
    // free flight and for the BF16 / FP8 stencil gather (mrp_params)
    void SetTracerFilter(bool hardware) { params.tracer_filter = hardware ? 1 : 0; push(); }
    void SetGatherFilter(bool hardware) { params.gather_filter = hardware ? 1 : 0; push(); }
    void SetMaxDensity(float md) {
        mrpnn::check(mrp_volume_set_max_density(h, md), "SetMaxDensity");
        max_density = md;
    }

    // core/volume.cu:487-548: sampleNum launches with the running mean;
    // RGB + (coverage for PT, hit distance for MRPNN).
    std::vector<float4> Render(int2 size, float3 ori, float3 up, float3 right, float3 lightDir,
                               RenderType rt = RenderType::PT, float g = 0.857f, float alpha = 1.0f,
                               float3 lightColor = {1, 1, 1}, int multiScatter = 512, int sampleNum = 1024) {
        mrp_view v = make_view(size, ori, up, right, lightDir, g, alpha, lightColor, multiScatter);
        std::vector<float4> out((size_t)size.x * size.y);
        mrpnn::check(mrp_render(h, &v, (mrp_render_type)rt, sampleNum, reinterpret_cast<float*>(out.data()), 0),
                     "Render");
        return out;
    }

    mrp_volume* handle() const { return h; }
    int Resolution() const { return resolution; }

   private:
    void push() { mrpnn::check(mrp_set_params(h, &params), "set params"); }
    mrp_view make_view(int2 size, float3 ori, float3 up, float3 right, float3 lightDir, float g, float alpha,
                       float3 lightColor, int multiScatter) {
        mrp_view v{};
        v.width = size.x;
        v.height = size.y;
        v.ori[0] = ori.x; v.ori[1] = ori.y; v.ori[2] = ori.z;
        v.up[0] = up.x; v.up[1] = up.y; v.up[2] = up.z;
        v.right[0] = right.x; v.right[1] = right.y; v.right[2] = right.z;
        v.light_dir[0] = lightDir.x; v.light_dir[1] = lightDir.y; v.light_dir[2] = lightDir.z;
        v.light_color[0] = lightColor.x; v.light_color[1] = lightColor.y; v.light_color[2] = lightColor.z;
        v.alpha = alpha;
        v.g = g;
        v.multi_scatter = multiScatter;
        v.spp = 32;   // RenderCamera<false> traces 32 samples per launch (core/volume.cu:222)
        v.seed = 0;
        v.frame_offset = 0;
        return v;
    }

    int resolution;
    mrp_volume* h = nullptr;
    mrp_params params;
    std::vector<float> datas;
    bool dirty = true;
    bool checkboard = true;
    float exposure = 1.0f, ior = -1.0f;
    std::vector<float> lut_host;
    float lut_host_g = 0.0f;
};

typedef std::function<float3(float3 radiance)> ToneMapFunction;

namespace mrpnn {
// Minimal PNG writer (8-bit RGBA, stored deflate blocks; CRC-32 and
// Adler-32 as in RFC 1950/1951 and the PNG specification).
inline uint32_t crc32(const uint8_t* p, size_t n, uint32_t c = 0xFFFFFFFFu) {
    for (size_t i = 0; i < n; ++i) {
        c ^= p[i];
        for (int k = 0; k < 8; ++k) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
    }
    return c;
}
inline bool write_png_rgba(const std::string& path, const uint8_t* rgba, int w, int h) {
    std::vector<uint8_t> raw;
    raw.reserve((size_t)h * (w * 4 + 1));
    for (int y = 0; y < h; ++y) {
        raw.push_back(0);
        raw.insert(raw.end(), rgba + (size_t)y * w * 4, rgba + (size_t)(y + 1) * w * 4);
    }
    std::vector<uint8_t> z = {0x78, 0x01};
    uint32_t a = 1, b = 0;
    for (uint8_t c : raw) { a = (a + c) % 65521u; b = (b + a) % 65521u; }
    for (size_t off = 0; off < raw.size() || off == 0; off += 65535) {
        size_t len = std::min<size_t>(65535, raw.size() - off);
        z.push_back(off + len >= raw.size() ? 1 : 0);
        z.push_back((uint8_t)(len & 0xFF)); z.push_back((uint8_t)(len >> 8));
        z.push_back((uint8_t)(~len & 0xFF)); z.push_back((uint8_t)((~len >> 8) & 0xFF));
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
        if (raw.empty()) break;
    }
    uint32_t adler = (b << 16) | a;
    for (int s = 24; s >= 0; s -= 8) z.push_back((uint8_t)(adler >> s));
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    auto be32 = [&](uint32_t v) { uint8_t q[4] = {(uint8_t)(v >> 24), (uint8_t)(v >> 16), (uint8_t)(v >> 8), (uint8_t)v}; std::fwrite(q, 1, 4, f); };
    auto chunk = [&](const char* type, const std::vector<uint8_t>& data) {
        be32((uint32_t)data.size());
        std::vector<uint8_t> td(type, type + 4);
        td.insert(td.end(), data.begin(), data.end());
        std::fwrite(td.data(), 1, td.size(), f);
        be32(crc32(td.data(), td.size()) ^ 0xFFFFFFFFu);
    };
    const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    std::fwrite(sig, 1, 8, f);
    std::vector<uint8_t> ihdr = {(uint8_t)(w >> 24), (uint8_t)(w >> 16), (uint8_t)(w >> 8), (uint8_t)w,
                                 (uint8_t)(h >> 24), (uint8_t)(h >> 16), (uint8_t)(h >> 8), (uint8_t)h, 8, 6, 0, 0, 0};
    chunk("IHDR", ihdr);
    chunk("IDAT", z);
    chunk("IEND", {});
    return std::fclose(f) == 0;
}
}  // namespace mrpnn

class Camera {
   public:
    int resolution;
    std::string name;

    static float3 Gamma(float3 c) {
        return float3{std::pow(c.x, 1.0f / 2.2f), std::pow(c.y, 1.0f / 2.2f), std::pow(c.z, 1.0f / 2.2f)};
    }
    // The ACES fit belongs to the interactive frame path (not built yet);
    // RenderToFile ignores its tone argument, as the reference does.
    static float3 ACES(float3 c) { return Gamma(c); }
    static float3 None(float3 c) { return c; }

    // core/camera.cu:166-192
    Camera(VolumeRender& volume, std::string name = "test camera", float3 position = {0.75f, 0.75f, 0.75f},
           int resolution = 512)
        : resolution(resolution), name(name), volume(&volume) {
        SetPosition(position);
    }
    void SetPosition(float3 position) {
        ori = position;
        float l = std::sqrt(ori.x * ori.x + ori.y * ori.y + ori.z * ori.z);
        forward = float3{-ori.x / l, -ori.y / l, -ori.z / l};
        // right = normalize(cross((0,1,0), forward)); up = cross(forward, right)
        float3 r{forward.z, 0.0f, -forward.x};
        float rl = std::sqrt(r.x * r.x + r.y * r.y + r.z * r.z);
        right = float3{r.x / rl, r.y / rl, r.z / rl};
        up = float3{forward.y * right.z - forward.z * right.y, forward.z * right.x - forward.x * right.z,
                    forward.x * right.y - forward.y * right.x};
        if (position.x == 0 && position.z == 0) {
            right = float3{1, 0, 0};
            up = position.y > 0 ? float3{0, 0, 1} : float3{0, 0, -1};
        }
    }
    float3 GetPosition() const { return ori; }
    void SetVolume(VolumeRender& v) { volume = &v; }

    // core/camera.cu:198-226: the reference's body is commented out.
    void Render(float3, float3 = {1, 1, 1}, float = 1, int = 1, float = 0, int = 1, ToneMapFunction = ACES,
                VolumeRender::RenderType = VolumeRender::RenderType::PT, float = 1.0f) {}

    // core/camera.cu:229-257: render, saturate to 8 bit, write path + ".png".
    void RenderToFile(std::string path, float3 lightDir, float3 lightColor = {1, 1, 1}, float alpha = 1,
                      int multiScatter = 1, float g = 0, int sampleNum = 1, ToneMapFunction /*tone*/ = ACES,
                      VolumeRender::RenderType rt = VolumeRender::RenderType::PT, float /*exp*/ = 1.0f) {
        auto res = volume->Render(int2{resolution, resolution}, ori, up, right, lightDir, rt, g, alpha, lightColor,
                                  multiScatter, sampleNum);
        std::vector<uint8_t> data((size_t)resolution * resolution * 4);
        auto sat = [](float v) { return v < 0 ? 0.0f : (v > 1 ? 1.0f : v); };
        for (size_t i = 0; i < res.size(); ++i) {
            data[4 * i] = (uint8_t)(sat(res[i].x) * 255);
            data[4 * i + 1] = (uint8_t)(sat(res[i].y) * 255);
            data[4 * i + 2] = (uint8_t)(sat(res[i].z) * 255);
            data[4 * i + 3] = 255;
        }
        if (!mrpnn::write_png_rgba(path + ".png", data.data(), resolution, resolution))
            throw mrpnn::Error(MRP_ERR_IO, "RenderToFile: cannot write " + path + ".png");
    }

   protected:
    float3 ori, forward, right, up;
    VolumeRender* volume;
};
