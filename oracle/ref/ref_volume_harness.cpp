// ref_volume_harness.cpp -- C entry points over the reference's volume
// builders in core/volume.cu, compiled on the CPU (oracle/Makefile `ref`
// target -> oracle/_ref/libmrpnn_ref_volume.so).
//
// TEST INFRASTRUCTURE ONLY.  It pins the oracle's restatements of
// VolumeRender::Update's CPU pyramid (core/volume.cu:835-882, 1443-1531),
// Update_TR with Fill_TR (:1533-1560, 1589-1667), Fill_Hg and its scrambled
// radical inverse (:1186-1400), GetHGLut (:1424-1442), Fill_BakeTR
// (:1562-1587) and the RGBE loader behind SetHDRI (core/hdr_loader.h,
// core/volume.cu:1696-1728).  The recipe compiles a build copy of
// core/volume.cu in which each `K<<<grid, block>>>(args);` statement is
// rewritten to `ref_launch(grid, block, [&] { K(args); });` (every other byte
// as it is); the reference's classes and functions run unmodified, with the
// CUDA runtime replaced by shim/ref_runtime.h.
#include <mutex>

#include "volume_gcc.cu"

#include "ref_support.h"

// VolumeRender keeps its host copies and arrays private.  An explicit
// template instantiation may name private members (access is not checked
// there), which lets this harness read what Update / Update_TR produced
// without changing the class.
template <class Tag>
struct Member {
    static typename Tag::type ptr;
};
template <class Tag>
typename Tag::type Member<Tag>::ptr;
template <class Tag, typename Tag::type P>
struct Bind {
    Bind() { Member<Tag>::ptr = P; }
    static Bind instance;
};
template <class Tag, typename Tag::type P>
Bind<Tag, P> Bind<Tag, P>::instance;

struct M_datas { using type = float* VolumeRender::*; };
struct M_mips { using type = float* (VolumeRender::*)[9]; };
struct M_tr_mips { using type = float* (VolumeRender::*)[8]; };
struct M_mips_dev { using type = cudaArray* (VolumeRender::*)[9]; };
struct M_mip_size { using type = cudaExtent (VolumeRender::*)[9]; };
struct M_tr_mips_dev { using type = cudaArray* (VolumeRender::*)[8]; };
struct M_datas_dev { using type = cudaArray* VolumeRender::*; };
struct M_datas_devL { using type = cudaArray* VolumeRender::*; };
struct M_datas_devS { using type = cudaArray* VolumeRender::*; };
struct M_hglut { using type = float* VolumeRender::*; };
struct M_hglut_dev { using type = cudaArray* VolumeRender::*; };
struct M_tr_lightDir { using type = float3 VolumeRender::*; };
struct M_tr_alpha { using type = float VolumeRender::*; };
struct M_hginlut { using type = float VolumeRender::*; };
template struct Bind<M_datas, &VolumeRender::datas>;
template struct Bind<M_mips, &VolumeRender::mips>;
template struct Bind<M_tr_mips, &VolumeRender::tr_mips>;
template struct Bind<M_mips_dev, &VolumeRender::mips_dev>;
template struct Bind<M_mip_size, &VolumeRender::mip_size>;
template struct Bind<M_tr_mips_dev, &VolumeRender::tr_mips_dev>;
template struct Bind<M_datas_dev, &VolumeRender::datas_dev>;
template struct Bind<M_datas_devL, &VolumeRender::datas_devL>;
template struct Bind<M_datas_devS, &VolumeRender::datas_devS>;
template struct Bind<M_hglut, &VolumeRender::hglut>;
template struct Bind<M_hglut_dev, &VolumeRender::hglut_dev>;
template struct Bind<M_tr_lightDir, &VolumeRender::tr_lightDir>;
template struct Bind<M_tr_alpha, &VolumeRender::tr_alpha>;
template struct Bind<M_hginlut, &VolumeRender::hginlut>;

template <class Tag>
static auto& mem(VolumeRender* v) {
    return v->*Member<Tag>::ptr;
}

// VolumeRender(int) in zeroed storage.  The int constructor leaves members
// such as tr_lightDir uninitialised (LoadData sets them, core/volume.cu:
// 973-975); they are set here as LoadData does, so that Update_TR never
// skips its work on a stale match.
static VolumeRender* new_volume(int R) {
    VolumeRender* v = new (std::calloc(1, sizeof(VolumeRender))) VolumeRender(R);
    mem<M_tr_lightDir>(v) = float3{FLT_MAX, FLT_MAX, FLT_MAX};
    mem<M_tr_alpha>(v) = -1.0f;
    mem<M_hginlut>(v) = -100.0f;
    return v;
}

// ... with its data set and Update() run.  The int constructor does not
// allocate datas_dev and mips_dev either (the file loader does, core/
// volume.cu:978-1058); they are allocated here as the loader would, with the
// density array at the volume's own resolution.
static VolumeRender* make_volume(const float* data, int R, float max_density) {
    VolumeRender* v = new_volume(R);
    cudaChannelFormatDesc desc = cudaCreateChannelDesc<float>();
    cudaMalloc3DArray(&mem<M_datas_dev>(v), &desc, cudaExtent{(size_t)R, (size_t)R, (size_t)R});
    for (int i = 0; i < 9; ++i) cudaMalloc3DArray(&mem<M_mips_dev>(v)[i], &desc, mem<M_mip_size>(v)[i]);
    std::memcpy(mem<M_datas>(v), data, sizeof(float) * (size_t)R * R * R);
    v->max_density = max_density;
    v->Update(true, true);
    return v;
}

// The reference's texture and surface references are globals; after a
// volume is freed none may still point into its arrays.
static void unbind_all() {
    surfRef.array = nullptr;
    hgSurfRef.array = nullptr;
    texRef.data = nullptr;
    _DensityVolume.data = nullptr;
    _HGLut.data = nullptr;
    texture<float, cudaTextureType3D, cudaReadModeElementType>* t[17] = {
        &_Mips0, &_Mips1, &_Mips2, &_Mips3, &_Mips4, &_Mips5, &_Mips6, &_Mips7, &_Mips8,
        &_TR_Mips0, &_TR_Mips1, &_TR_Mips2, &_TR_Mips3, &_TR_Mips4, &_TR_Mips5, &_TR_Mips6, &_TR_Mips7};
    for (auto* x : t) x->data = nullptr;
}

// Frees what make_volume and the constructor allocated.  The reference's
// destructor is not run: it also frees dataCache[i].mips_dev[i], pointers
// the int constructor never initialises (core/volume.cu:1172-1175).
static void drop_volume(VolumeRender* v) {
    cudaFreeArray(mem<M_datas_dev>(v));
    cudaFreeArray(mem<M_datas_devL>(v));
    cudaFreeArray(mem<M_datas_devS>(v));
    cudaFreeArray(mem<M_hglut_dev>(v));
    for (int i = 0; i < 9; ++i) {
        cudaFreeArray(mem<M_mips_dev>(v)[i]);
        delete[] mem<M_mips>(v)[i];
    }
    for (int i = 0; i < 8; ++i) {
        cudaFreeArray(mem<M_tr_mips_dev>(v)[i]);
        delete[] mem<M_tr_mips>(v)[i];
    }
    delete[] mem<M_datas>(v);
    delete[] mem<M_hglut>(v);
    std::free(v);
    unbind_all();
}

extern "C" {

// VolumeRender::Update(true, true): the 9-level pyramid built on the CPU
// (mips_out: levels 256>>m concatenated).
void ref_vol_pyramid(const float* data, int R, float* mips_out) {
    VolumeRender* v = make_volume(data, R, 1.0f);
    size_t off = 0;
    for (int m = 0; m < 9; ++m) {
        size_t n = (size_t)(256 >> m) * (256 >> m) * (256 >> m);
        std::memcpy(mips_out + off, mem<M_mips>(v)[m], n * sizeof(float));
        off += n;
    }
    drop_volume(v);
}

// VolumeRender::Update_TR(lightDir, alpha, CPU): cpu = 0 runs the device
// branch (Fill_TR over the mip arrays, the path the renderer takes), cpu = 1
// the host branch (Sample_TR); tr_out: levels 128>>i concatenated.
void ref_vol_tr(const float* data, int R, float alpha, const float L[3], int cpu, float* tr_out) {
    VolumeRender* v = make_volume(data, R, 1.0f);
    v->Update_TR(float3{L[0], L[1], L[2]}, alpha, cpu != 0);
    size_t off = 0;
    for (int i = 0; i < 8; ++i) {
        size_t n = (size_t)(128 >> i) * (128 >> i) * (128 >> i);
        const float* src = cpu ? mem<M_tr_mips>(v)[i] : (const float*)mem<M_tr_mips_dev>(v)[i]->mem();
        std::memcpy(tr_out + off, src, n * sizeof(float));
        off += n;
    }
    drop_volume(v);
}

// Fill_Hg for a list of texels (index j * 512 + i: row j = cone angle,
// column i = cos theta).  Each texel runs as its own thread of the kernel's
// 8 x 8 blocks; its one random draw (the shift bn) comes from Philox stream
// (kind 1, id texel, sub 0, frame 0, seed), the stream the oracle and the
// kernels use for it.
void ref_vol_hg_texels(float g, uint32_t seed, const int* texels, int n, float* out) {
    hgSurfRef.array = nullptr;   // the texels are read back one at a time
    std::vector<std::thread> pool;
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    for (unsigned t = 0; t < nt; ++t) {
        pool.emplace_back([&, t] {
            blockDim = dim3(8, 8);
            gridDim = dim3(LUT_SIZE / 8, LUT_SIZE / 8);
            for (int q = (int)t; q < n; q += (int)nt) {
                unsigned i = (unsigned)(texels[q] % LUT_SIZE), j = (unsigned)(texels[q] / LUT_SIZE);
                blockIdx = uint3{i / 8, j / 8, 0};
                threadIdx = uint3{i % 8, j % 8, 0};
                ref_set_stream(1, (uint32_t)texels[q], 0, 0, seed);
                Fill_Hg(g);
                out[q] = ref_last_surface_value;
            }
        });
    }
    for (auto& th : pool) th.join();
}

// VolumeRender::GetHGLut(cos, angle) over the host table `lut` (512 x 512).
float ref_vol_get_hg_lut(const float* lut, float cosv, float angle) {
    static VolumeRender* v = nullptr;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (!v) v = new_volume(2);
    std::memcpy(mem<M_hglut>(v), lut, sizeof(float) * LUT_SIZE * LUT_SIZE);
    return v->GetHGLut(cosv, angle);
}

// Fill_BakeTR for a list of voxels (index (x * B + y) * B + z of the B^3
// bake grid) of the volume `data` (R^3, majorant max_density): each voxel is
// one thread; its estimates draw Philox stream (kind 2, id voxel, sub 0,
// frame 0, seed), restarted by the kernel's InitRand before each estimate.
void ref_vol_bake_voxels(const float* data, int R, float max_density, float alpha, const float L[3], int bake_res,
                         uint32_t seed, const int64_t* voxels, int n, float* out) {
    VolumeRender* v = make_volume(data, R, max_density);
    surfRef.array = nullptr;   // the estimates are read back one voxel at a time
    std::vector<std::thread> pool;
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    for (unsigned t = 0; t < nt; ++t) {
        pool.emplace_back([&, t] {
            blockDim = dim3(1, 1, 1);
            gridDim = dim3(bake_res, bake_res, bake_res);
            threadIdx = uint3{0, 0, 0};
            for (int q = (int)t; q < n; q += (int)nt) {
                int64_t vi = voxels[q];
                unsigned x = (unsigned)(vi / ((int64_t)bake_res * bake_res));
                unsigned y = (unsigned)((vi / bake_res) % bake_res), z = (unsigned)(vi % bake_res);
                blockIdx = uint3{x, y, z};
                ref_set_stream(2, (uint32_t)vi, (uint32_t)(vi >> 32) * 8u, 0, seed);
                Fill_BakeTR(bake_res, alpha, float3{L[0], L[1], L[2]});
                out[q] = ref_last_surface_value;
            }
        });
    }
    for (auto& th : pool) th.join();
    drop_volume(v);
}

// The reference's RGBE loader (core/hdr_loader.h load_hdr_float4, as
// SetHDRI calls it): 0 on success; the size into rx, ry and, when out holds
// at least rx * ry * 4 floats (out_floats), the RGBA pixels.
int ref_vol_load_hdr(const char* path, unsigned* rx, unsigned* ry, float* out, size_t out_floats) {
    float* px = nullptr;
    if (!load_hdr_float4(&px, rx, ry, path)) return 1;
    size_t n = (size_t)*rx * *ry * 4;
    if (out && out_floats >= n) std::memcpy(out, px, n * sizeof(float));
    std::free(px);
    return 0;
}

// The viewer's PT frame (RenderCamera<false> with the histogram buffer,
// core/volume.cu:57-150) over a scene bound as Update / Update_CachedTR bind
// it: density (border), the baked NEE grid as _TR_Mips0 (clamp), majorant,
// albedo, constant sky.  Pixel (row i, column j) runs as the kernel's thread
// (i, column slot) with its random numbers from Philox stream (0, i W + j, 0,
// frame, seed); frame_num is the kernel's frameNum (its running-mean count).
void ref_vol_frame_pt(const float* density, int R, float max_density, const float* baked, int baked_res,
                      const float sr[3], const float sky[3], int W, int H, const float ori[3], const float up[3],
                      const float right[3], const float L[3], const float lc[3], float alpha, float g, int multi,
                      uint32_t seed, int frame, int frame_num, int checker, int flip_, float* target, float* histo) {
    _DensityVolume.data = density;
    _DensityVolume.nx = _DensityVolume.ny = _DensityVolume.nz = R;
    _DensityVolume.addressMode[0] = _DensityVolume.addressMode[1] = _DensityVolume.addressMode[2] =
        cudaAddressModeBorder;
    _TR_Mips0.data = baked;
    _TR_Mips0.nx = _TR_Mips0.ny = _TR_Mips0.nz = baked_res;
    _TR_Mips0.addressMode[0] = _TR_Mips0.addressMode[1] = _TR_Mips0.addressMode[2] = cudaAddressModeClamp;
    Resolution = R;
    maxDensity = max_density;
    scatter_rate = float3{sr[0], sr[1], sr[2]};
    tr_scale = 1.0f;
    enviroment_exp = 1.0f;
    _HDRI.data = nullptr;
    _HDRI.constant = float4{sky[0], sky[1], sky[2], 1.0f};
    dev_checkboard = checker;
    flip = flip_;
    frameNum = frame_num;
    const int cols = checker ? (W + 1) / 2 : W;
    std::vector<std::thread> pool;
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    for (unsigned t = 0; t < nt; ++t) {
        pool.emplace_back([&, t] {
            blockDim = dim3(1, 1, 1);
            threadIdx = uint3{0, 0, 0};
            for (int q = (int)t; q < H * cols; q += (int)nt) {
                int i = q / cols, jj = q % cols;
                int j = checker ? jj * 2 + ((i + flip_) % 2) : jj;
                if (j >= W) continue;
                blockIdx = uint3{(unsigned)i, (unsigned)jj, 0};
                ref_set_stream(0, (uint32_t)(i * W + j), 0, (uint32_t)frame, seed);
                RenderCamera<false>(reinterpret_cast<float3*>(target), reinterpret_cast<Histogram*>(histo),
                                    int2{W, H}, float3{ori[0], ori[1], ori[2]}, float3{up[0], up[1], up[2]},
                                    float3{right[0], right[1], right[2]}, float3{L[0], L[1], L[2]},
                                    float3{lc[0], lc[1], lc[2]}, alpha, multi, g);
            }
        });
    }
    for (auto& th : pool) th.join();
    _DensityVolume.data = nullptr;
    _TR_Mips0.data = nullptr;
}

// The viewer's finishing pass: Denoise<denoise> for a PT frame or
// ReprojectionDenoise for a predictor frame (core/volume.cu:285-372, the
// tone maps of core/ACES.cuh), RGBA8 into rgba8.
void ref_vol_frame_finish(float* target, float* histo, int W, int H, int frame_num, int flip_, int predict, int denoise,
                          float exposure_, int tone, uint32_t* rgba8) {
    frameNum = frame_num;
    flip = flip_;
    exposure = exposure_;
    blockDim = dim3(1, 1, 1);
    threadIdx = uint3{0, 0, 0};
    for (int id = 0; id < W * H; ++id) {
        blockIdx = uint3{(unsigned)id, 0, 0};
        float3* T = reinterpret_cast<float3*>(target);
        Histogram* Hs = reinterpret_cast<Histogram*>(histo);
        if (predict) ReprojectionDenoise(T, Hs, rgba8, int2{W, H}, tone);
        else if (denoise) Denoise<true>(T, Hs, rgba8, int2{W, H}, tone);
        else Denoise<false>(T, Hs, rgba8, int2{W, H}, tone);
    }
}

// The pieces of Render's light choice with an environment map
// (core/volume.cu:494-509): Roberts2, UniformSampleSphere and
// Image_host::Sample.
void ref_vol_roberts2(int n, float out[3]) {
    float3 r = Roberts2(n);
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void ref_vol_uniform_sample_sphere(float ex, float ey, float out[3]) {
    float3 d = UniformSampleSphere(float2{ex, ey});
    out[0] = d.x; out[1] = d.y; out[2] = d.z;
}
void ref_vol_image_sample(const float* rgba, int sx, int sy, float u, float v, float out[3]) {
    Image_host img;
    img.data = reinterpret_cast<float4*>(const_cast<float*>(rgba));
    img.sx = sx;
    img.sy = sy;
    float3 c = img.Sample(float2{u, v});
    img.data = nullptr;
    out[0] = c.x; out[1] = c.y; out[2] = c.z;
}

}  // extern "C"
