// hdri.cu -- the environment map of VolumeRender::SetHDRI (core/volume.cu:
// 1696-1728): Radiance RGBE (.hdr) files read on the host, the map kept on
// the device for SkyBox (sky_radiance in common.cuh) and on the host for the
// light sampling of the predictor's launches (core/volume.cu:494-509).
//
// File format (the reader of core/hdr_loader.h): a first line starting with
// "#?", header lines up to the resolution line ("-Y <h> +X <w>"; '#' lines
// and unknown lines skipped; FORMAT must be 32-bit_rle_rgbe or
// 32-bit_rle_xyze; EXPOSURE / GAMMA are read and not applied), then h
// scanlines of w RGBE pixels, each flat or, for 8 <= w <= 0x7fff, in the
// new-style run-length encoding (2, 2, w >> 8, w & 255, then per component
// runs: a count byte > 128 repeats the next byte count - 128 times, else
// count literal bytes follow).  Mantissa m and exponent e give
// (m + 0.5) * 2^(e - 136) per channel (the exponent field is built as
// ((e - 9) << 23) & 0x7f800000, as the reference does); e = 0 is black;
// alpha is 0.  Rows are stored top to bottom as they appear in the file.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "abi_internal.h"

using namespace mrpi;

namespace {

constexpr unsigned kMaxEdge = 1u << 15;

struct File {
    FILE* f = nullptr;
    explicit File(const char* p) : f(std::fopen(p, "rb")) {}
    ~File() { if (f) std::fclose(f); }
};

bool starts(const char* line, const char* id) { return std::strncmp(line, id, std::strlen(id)) == 0; }

mrp_status read_header(FILE* f, const char* path, unsigned* w, unsigned* h) {
    char line[2048];
    if (!std::fgets(line, sizeof line, f)) return fail(MRP_ERR_IO, "%s: empty file", path);
    if (line[0] != '#' && line[1] != '?') return fail(MRP_ERR_IO, "%s: not a Radiance .hdr file", path);
    for (;;) {
        if (!std::fgets(line, sizeof line, f)) return fail(MRP_ERR_IO, "%s: no resolution line", path);
        if (line[0] == '#') continue;
        if (starts(line, "FORMAT=")) {
            const char* c = line + 7;
            if (!starts(c, "32-bit_rle_rgbe") && !starts(c, "32-bit_rle_xyze"))
                return fail(MRP_ERR_IO, "%s: unsupported FORMAT", path);
        } else if (line[0] == '-' || line[0] == '+') {
            const char* x = std::strchr(line, 'X');
            const char* y = std::strchr(line, 'Y');
            if (!x || x <= line || std::sscanf(x + 1, "%u", w) != 1 || !y || y <= line ||
                std::sscanf(y + 1, "%u", h) != 1)
                return fail(MRP_ERR_IO, "%s: bad resolution line", path);
            if (*w == 0 || *h == 0 || *w > kMaxEdge || *h > kMaxEdge)
                return fail(MRP_ERR_IO, "%s: image size %ux%u", path, *w, *h);
            return MRP_OK;
        }
    }
}

bool read_flat(FILE* f, unsigned char* buf, unsigned n) { return std::fread(buf, 4, n, f) == n; }

// One scanline of w RGBE pixels into buf (4 w bytes).
mrp_status read_scanline(FILE* f, const char* path, unsigned char* buf, unsigned w, bool rle) {
    if (!rle) return read_flat(f, buf, w) ? MRP_OK : fail(MRP_ERR_IO, "%s: truncated pixels", path);
    int c = std::fgetc(f);
    if (c == EOF) return fail(MRP_ERR_IO, "%s: truncated pixels", path);
    if (c != 2) {   // a flat scanline
        std::ungetc(c, f);
        return read_flat(f, buf, w) ? MRP_OK : fail(MRP_ERR_IO, "%s: truncated pixels", path);
    }
    int g = std::fgetc(f), b = std::fgetc(f), e = std::fgetc(f);
    if (g == EOF || b == EOF || e == EOF) return fail(MRP_ERR_IO, "%s: truncated pixels", path);
    if (g != 2 || (b & 128)) {   // a flat scanline whose first pixel starts with 2
        buf[0] = 2; buf[1] = (unsigned char)g; buf[2] = (unsigned char)b; buf[3] = (unsigned char)e;
        return read_flat(f, buf + 4, w - 1) ? MRP_OK : fail(MRP_ERR_IO, "%s: truncated pixels", path);
    }
    if ((unsigned)(b << 8 | e) != w) return fail(MRP_ERR_IO, "%s: scanline length mismatch", path);
    for (int ch = 0; ch < 4; ++ch) {
        for (unsigned pos = 0; pos < w;) {
            int n = std::fgetc(f);
            if (n == EOF) return fail(MRP_ERR_IO, "%s: truncated run", path);
            if (n > 128) {
                n &= 127;
                int v = std::fgetc(f);
                if (v == EOF || pos + n > w) return fail(MRP_ERR_IO, "%s: bad run", path);
                for (int k = 0; k < n; ++k) buf[4 * pos++ + ch] = (unsigned char)v;
            } else {
                if (n == 0 || pos + n > w) return fail(MRP_ERR_IO, "%s: bad run", path);
                for (int k = 0; k < n; ++k) {
                    int v = std::fgetc(f);
                    if (v == EOF) return fail(MRP_ERR_IO, "%s: truncated run", path);
                    buf[4 * pos++ + ch] = (unsigned char)v;
                }
            }
        }
    }
    return MRP_OK;
}

void rgbe_to_rgba(const unsigned char* p, float* out) {
    if (p[3] == 0) {
        out[0] = out[1] = out[2] = 0.0f;
    } else {
        uint32_t bits = (uint32_t)(((int)p[3] - 9) << 23) & 0x7f800000u;
        float s;
        std::memcpy(&s, &bits, 4);
        out[0] = ((float)p[0] + 0.5f) * s;
        out[1] = ((float)p[1] + 0.5f) * s;
        out[2] = ((float)p[2] + 0.5f) * s;
    }
    out[3] = 0.0f;
}

}  // namespace

namespace mrpi {

// The light of one predictor launch with an environment map set
// (core/volume.cu:494-509): with probability rate = 4 env_exp / (4 env_exp +
// max(light colour)) the map itself lights the launch, from the direction
// UniformSampleSphere(Roberts2(n)) with the colour Image_host::Sample(uv)
// * env_exp * 4 / rate (bilinear, clamp addressing); otherwise the light
// colour is divided by 1 - rate.  coin is the launch's uniform draw (the
// reference calls rand()).
void hdri_light(const mrp_volume* v, float coin, int n, float L[3], float C[3]) {
    const float e4 = v->params.env_exp * 4.0f;
    const float rate = e4 / (e4 + std::fmax(C[0], std::fmax(C[1], C[2])));
    if (!(coin < rate)) {
        for (int c = 0; c < 3; ++c) C[c] = C[c] / (1.0f - rate);
        return;
    }
    // Roberts2 (core/vector.cu:179-183)
    const float g = 1.32471795724474602596f;
    const float ax = 1.0f / g, ay = 1.0f / (g * g);
    auto frac = [](float f) { return f - (float)(long)f; };
    const float ex = frac(ax * (float)n + 0.5f), ey = frac(ay * (float)n + 0.5f);
    // UniformSampleSphere (core/vector.cu:195-205)
    const float phi = 2 * 3.14159265359f * ex;
    const float ct = 1 - 2 * ey;
    const float stt = std::sqrt(1 - ct * ct);
    const float d[3] = {stt * std::cos(phi), stt * std::sin(phi), ct};
    const float u = atan2f(-d[2], d[0]) * (float)(0.5 / 3.1415926) + 0.5f;
    const float w = acosf(std::fmax(std::fmin(d[1], 1.0f), -1.0f)) * (float)(1.0 / 3.1415926);
    // Image_host::Sample (core/volume.hpp:24-42)
    const int W = v->hdri_w, H = v->hdri_h;
    const float px = u * (float)W - 0.5f, py = w * (float)H - 0.5f;
    const int x = (int)std::floor(px), y = (int)std::floor(py);
    const float wx = px - (float)x, wy = py - (float)y;
    auto S = [&](int a, int b, int c) {
        a = a < 0 ? 0 : (a > W - 1 ? W - 1 : a);
        b = b < 0 ? 0 : (b > H - 1 ? H - 1 : b);
        return v->hdri_host[4 * ((size_t)b * W + a) + c];
    };
    auto lerp = [](float a, float b, float t) { return a * (1.0f - t) + b * t; };
    for (int c = 0; c < 3; ++c) {
        float s = lerp(lerp(S(x, y, c), S(x + 1, y, c), wx), lerp(S(x, y + 1, c), S(x + 1, y + 1, c), wx), wy);
        C[c] = s * v->params.env_exp * 4.0f / rate;
        L[c] = d[c];
    }
}

}  // namespace mrpi

extern "C" {

mrp_status mrp_hdri_file_read(const char* path, int* width, int* height, float* rgba, size_t rgba_floats) {
    if (!path || !width || !height) return fail(MRP_ERR_INVALID, "null argument");
    File F(path);
    if (!F.f) return fail(MRP_ERR_IO, "cannot open %s", path);
    unsigned w = 0, h = 0;
    TRY(read_header(F.f, path, &w, &h));
    *width = (int)w;
    *height = (int)h;
    if (!rgba) return MRP_OK;
    if (rgba_floats < (size_t)w * h * 4)
        return fail(MRP_ERR_INVALID, "%s: buffer holds %zu of %zu floats", path, rgba_floats, (size_t)w * h * 4);
    const bool rle = !(w < 8 || w > 0x7fff);
    std::vector<unsigned char> line((size_t)w * 4);
    for (unsigned j = 0; j < h; ++j) {
        TRY(read_scanline(F.f, path, line.data(), w, rle));
        for (unsigned i = 0; i < w; ++i) rgbe_to_rgba(&line[4 * i], rgba + 4 * ((size_t)j * w + i));
    }
    return MRP_OK;
}

mrp_status mrp_volume_set_hdri(mrp_volume* v, const float* rgba, int width, int height) {
    TRY(need_init());
    if (!v) return fail(MRP_ERR_INVALID, "null volume");
    if (rgba && (width < 1 || height < 1 || width > (int)kMaxEdge || height > (int)kMaxEdge))
        return fail(MRP_ERR_INVALID, "environment map size %dx%d", width, height);
    if (v->async_inflight) TRY(mrp_render_wait(v, 0));
    CU(cudaStreamSynchronize(v->stream));
    mrp::dev_free(v->hdri);
    v->hdri = nullptr;
    v->hdri_w = v->hdri_h = 0;
    v->hdri_host.clear();
    if (!rgba) return MRP_OK;
    const size_t n = (size_t)width * height;
    CU(mrp::dev_malloc(&v->hdri, n * sizeof(float4)));
    CU(cudaMemcpy(v->hdri, rgba, n * sizeof(float4), cudaMemcpyHostToDevice));
    v->hdri_host.assign(rgba, rgba + 4 * n);
    v->hdri_w = width;
    v->hdri_h = height;
    return MRP_OK;
}

mrp_status mrp_volume_load_hdri(mrp_volume* v, const char* path) {
    int w = 0, h = 0;
    TRY(mrp_hdri_file_read(path, &w, &h, nullptr, 0));
    std::vector<float> px((size_t)w * h * 4);
    TRY(mrp_hdri_file_read(path, &w, &h, px.data(), px.size()));
    return mrp_volume_set_hdri(v, px.data(), w, h);
}

}  // extern "C"
