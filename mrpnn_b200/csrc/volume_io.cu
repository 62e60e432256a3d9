// volume_io.cu -- volume files of the reference (VolumeRender(string path,
// bool cacheTR) -> LoadData, core/volume.cu:970-1149), host only:
//   .bin  int32 resolution R, then R^3 float32, z fastest (the cache format);
//   .txt  R, then R^3 whitespace-separated floats;
//   .vox  256^3 voxels, integers 0..255 scaled by 64/255, 64 per line, lines
//         starting with 'w', 'h' or 'd' are header lines.
// Negative values are kept (the SDF convention of the reference's tools:
// a negative density is a distance the tracers step over).
#include <cctype>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "abi_internal.h"

using namespace mrpi;

namespace {
bool ends_with(const std::string& s, const char* suf) {
    size_t n = std::strlen(suf);
    return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}
bool file_exists(const std::string& p) {
    FILE* f = std::fopen(p.c_str(), "rb");
    if (f) std::fclose(f);
    return f != nullptr;
}
constexpr int kMaxRes = 2048;

// The file actually read for `path`: the .bin itself, else the .bin cache the
// reference writes beside a .txt / .vox file, else the .txt / .vox file.
std::string resolve(const std::string& path) {
    if (ends_with(path, ".bin")) return path;
    if (file_exists(path + ".bin")) return path + ".bin";
    return path;
}

mrp_status read_bin(const std::string& p, int* res, float* dst, size_t cap) {
    FILE* f = std::fopen(p.c_str(), "rb");
    if (!f) return fail(MRP_ERR_IO, "cannot open %s", p.c_str());
    int R = 0;
    if (std::fread(&R, sizeof(int), 1, f) != 1 || R < 2 || R > kMaxRes) {
        std::fclose(f);
        return fail(MRP_ERR_IO, "%s: bad resolution header", p.c_str());
    }
    *res = R;
    size_t n = (size_t)R * R * R;
    if (dst) {
        if (cap < n) { std::fclose(f); return fail(MRP_ERR_INVALID, "%s: buffer holds %zu of %zu floats", p.c_str(), cap, n); }
        if (std::fread(dst, sizeof(float), n, f) != n) { std::fclose(f); return fail(MRP_ERR_IO, "%s: truncated", p.c_str()); }
    }
    std::fclose(f);
    return MRP_OK;
}

mrp_status read_txt(const std::string& p, int* res, float* dst, size_t cap) {
    FILE* f = std::fopen(p.c_str(), "r");
    if (!f) return fail(MRP_ERR_IO, "cannot open %s", p.c_str());
    int R = 0;
    if (std::fscanf(f, "%d", &R) != 1 || R < 2 || R > kMaxRes) {
        std::fclose(f);
        return fail(MRP_ERR_IO, "%s: bad resolution header", p.c_str());
    }
    *res = R;
    size_t n = (size_t)R * R * R;
    if (dst) {
        if (cap < n) { std::fclose(f); return fail(MRP_ERR_INVALID, "%s: buffer holds %zu of %zu floats", p.c_str(), cap, n); }
        for (size_t i = 0; i < n; ++i)
            if (std::fscanf(f, "%f", dst + i) != 1) { std::fclose(f); return fail(MRP_ERR_IO, "%s: truncated at %zu", p.c_str(), i); }
    }
    std::fclose(f);
    return MRP_OK;
}

mrp_status read_vox(const std::string& p, int* res, float* dst, size_t cap) {
    std::ifstream in(p);
    if (!in) return fail(MRP_ERR_IO, "cannot open %s", p.c_str());
    *res = 256;
    const size_t n = (size_t)256 * 256 * 256;
    if (!dst) return MRP_OK;
    if (cap < n) return fail(MRP_ERR_INVALID, "%s: buffer holds %zu of %zu floats", p.c_str(), cap, n);
    const float scale = (float)(64.0 / 255.0);
    size_t i = 0;
    std::string line;
    while (i < n && std::getline(in, line)) {
        if (line.empty()) continue;
        char c = line[0];
        if (c == 'w' || c == 'h' || c == 'd') continue;
        std::istringstream ss(line);
        int v;
        int k = 0;
        while (k < 64 && i < n && (ss >> v)) { dst[i++] = (float)v * scale; ++k; }
    }
    if (i < n) return fail(MRP_ERR_IO, "%s: %zu of %zu voxels", p.c_str(), i, n);
    return MRP_OK;
}

mrp_status read_any(const std::string& path, int* res, float* dst, size_t cap) {
    std::string p = resolve(path);
    if (ends_with(p, ".bin")) return read_bin(p, res, dst, cap);
    if (ends_with(p, "txt")) return read_txt(p, res, dst, cap);
    if (ends_with(p, "vox")) return read_vox(p, res, dst, cap);
    return fail(MRP_ERR_IO, "%s: not a .bin, .txt or .vox volume (and no %s.bin)", path.c_str(), path.c_str());
}

// Majorants the reference hard-codes for its four datasets (LoadData,
// core/volume.cu:982-1002); every other file gets the computed maximum.
float named_majorant(const std::string& path) {
    if (path.find("CLOUD0") != std::string::npos) return 510.416656f;
    if (path.find("CLOUD1") != std::string::npos) return 505.490356f;
    if (path.find("MODEL0") != std::string::npos) return 64.0000000f;
    if (path.find("MODEL1") != std::string::npos) return 23.8960018f;
    return 0.0f;
}
}  // namespace

extern "C" {

mrp_status mrp_volume_file_read(const char* path, int* res, float* dst, size_t dst_floats) {
    if (!path || !res) return fail(MRP_ERR_INVALID, "null argument");
    return read_any(path, res, dst, dst_floats);
}

mrp_status mrp_volume_file_write_bin(const char* path, const float* data, int res) {
    if (!path || !data || res < 2 || res > kMaxRes) return fail(MRP_ERR_INVALID, "bad argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(MRP_ERR_IO, "cannot write %s", path);
    size_t n = (size_t)res * res * res;
    bool ok = std::fwrite(&res, sizeof(int), 1, f) == 1 && std::fwrite(data, sizeof(float), n, f) == n;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? MRP_OK : fail(MRP_ERR_IO, "short write to %s", path);
}

mrp_status mrp_volume_load(const char* path, int write_cache, mrp_volume** out) {
    TRY(need_init());
    if (!path || !out) return fail(MRP_ERR_INVALID, "null argument");
    std::string p = path;
    int R = 0;
    TRY(read_any(p, &R, nullptr, 0));
    std::vector<float> data((size_t)R * R * R);
    TRY(read_any(p, &R, data.data(), data.size()));
    // the reference writes the .bin cache after parsing a .txt / .vox file
    std::string used = resolve(p);
    if (write_cache && !ends_with(used, ".bin")) TRY(mrp_volume_file_write_bin((p + ".bin").c_str(), data.data(), R));
    mrp_volume* v = nullptr;
    TRY(mrp_volume_create(R, &v));
    mrp_status st = mrp_volume_set_data(v, data.data(), R, 0);
    float md = named_majorant(p);
    if (st == MRP_OK && md > 0) st = mrp_volume_set_max_density(v, md);
    if (st == MRP_OK) st = mrp_volume_update(v, 1);
    if (st != MRP_OK) {
        mrp_volume_destroy(v);
        return st;
    }
    *out = v;
    return MRP_OK;
}

}  // extern "C"
