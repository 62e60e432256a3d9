// The reference's own usage (README "Use custom data": a sphere of radius
// 0.25 at the centre, Update, Render / Camera::RenderToFile) compiled against
// include/mrpnn_volume_render.hpp and run on libmrpnn_b200.so.
//
// usage: shim_example <out_prefix>   -> <out_prefix>.f32 (raw float4 frame), <out_prefix>.png,
//                                       <out_prefix>.fp16.f32 (the frame of an fp16-stored grid)
#include <cstdio>
#include <fstream>

#include "mrpnn_volume_render.hpp"

int main(int argc, char** argv) {
    std::string out = argc > 1 ? argv[1] : "shim_example";
    try {
        VolumeRender v(64);
        v.SetDatas([](int, int, int, float u, float w, float z) {
            float dx = u - 0.5f, dy = w - 0.5f, dz = z - 0.5f;
            return std::sqrt(dx * dx + dy * dy + dz * dz) < 0.25f ? 1.0f : 0.0f;
        });
        v.Update();
        v.SetScatterRate(0.99f);
        float3 L{0.3f, 0.8f, 0.5f};
        float n = std::sqrt(L.x * L.x + L.y * L.y + L.z * L.z);
        L = float3{L.x / n, L.y / n, L.z / n};
        Camera cam(v, "shim camera", float3{0.75f, 0.75f, 0.75f}, 64);
        cam.RenderToFile(out, L, float3{1, 1, 1}, 8.0f, 1, 0.857f, 1, Camera::ACES, VolumeRender::MRPNN);
        // the same frame through VolumeRender::Render, kept as raw floats
        float3 ori{0.75f, 0.75f, 0.75f};
        float3 fwd{-ori.x, -ori.y, -ori.z};
        float l = std::sqrt(fwd.x * fwd.x + fwd.y * fwd.y + fwd.z * fwd.z);
        fwd = float3{fwd.x / l, fwd.y / l, fwd.z / l};
        float3 r{fwd.z, 0.0f, -fwd.x};
        float rl = std::sqrt(r.x * r.x + r.z * r.z);
        r = float3{r.x / rl, 0.0f, r.z / rl};
        float3 u{fwd.y * r.z - fwd.z * r.y, fwd.z * r.x - fwd.x * r.z, fwd.x * r.y - fwd.y * r.x};
        auto img = v.Render(int2{64, 64}, ori, u, r, L, VolumeRender::MRPNN, 0.857f, 8.0f, float3{1, 1, 1}, 1, 2);
        std::ofstream(out + ".f32", std::ios::binary).write(reinterpret_cast<const char*>(img.data()),
                                                           img.size() * sizeof(float4));
        // the same volume with its device grid in fp16 (0 and 1 are exact)
        VolumeRender v16(64, MRP_STORAGE_FP16);
        v16.SetDatas([](int, int, int, float u, float w, float z) {
            float dx = u - 0.5f, dy = w - 0.5f, dz = z - 0.5f;
            return std::sqrt(dx * dx + dy * dy + dz * dz) < 0.25f ? 1.0f : 0.0f;
        });
        v16.Update();
        v16.SetScatterRate(0.99f);
        auto img16 = v16.Render(int2{64, 64}, ori, u, r, L, VolumeRender::MRPNN, 0.857f, 8.0f, float3{1, 1, 1}, 1, 2);
        std::ofstream(out + ".fp16.f32", std::ios::binary)
            .write(reinterpret_cast<const char*>(img16.data()), img16.size() * sizeof(float4));
        double s = 0;
        int hits = 0;
        for (auto& p : img) { s += p.x + p.y + p.z; hits += p.w > 0; }
        std::printf("shim_example: %d hit pixels, radiance sum %.6f, max density %.6f\n", hits, s, v.max_density);
    } catch (const mrpnn::Error& e) {
        std::fprintf(stderr, "shim_example: %s\n", e.what());
        return 2;
    }
    return 0;
}
