"""fp16 storage of the density grid (mrp_volume_create_ex, MRP_STORAGE_FP16)
against an fp32 volume holding the same fp16-rounded values.  Widening an
fp16 value to float is exact, so every derived resource (majorant, pyramid,
occupancy, TR levels, baked NEE grid) and every image (tracer, FP32 and BF16
predictor, batch rays) must agree bit for bit; the only inexact step is the
rounding on the way in, which must be IEEE round-to-nearest-even (numpy's
float16 conversion is the reference for it)."""
import ctypes as C

import numpy as np
import pytest

from tests.gpu_scene import LIGHT, view_frame

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _pair(R, seed=0, freq=4.0, bake_res=48):
    """An fp16 volume with a generated fBm grid and an fp32 volume set to its
    (widened) values; both updated, same parameters."""
    import mrpnn_b200 as M
    M.init()
    h = M.VolumeRender(R, storage="fp16")
    h.generate_fbm(seed, freq)
    f = M.VolumeRender(R)
    f.set_data(h.read(M.api.RES_DENSITY))
    for v in (h, f):
        v.Update()
        v.SetScatterRate(0.99)
        v.SetSky(0.05)
        v.SetBakeResolution(bake_res)
    return h, f


@pytest.fixture(scope="module")
def pair():
    return _pair(64)


def test_rounding_to_nearest_even():
    import torch

    import mrpnn_b200 as M
    M.init()
    R = 32
    rng = np.random.default_rng(3)
    x = rng.uniform(-3, 3, R ** 3).astype(np.float32)
    special = [0.0, -0.0, 1e-8, 3e-8, 6e-8, 5.9604645e-08, 1e-5, 0.1, 1 / 3, 2 / 3, 1.0, 1.0 + 2 ** -11,
               1.0 + 3 * 2 ** -11, 2048.5, 65504.0, 65519.0, 65520.0, 70000.0, -70000.0]
    x[:len(special)] = np.asarray(special, np.float32)
    with np.errstate(over="ignore"):
        ref = x.astype(np.float16).astype(np.float32)
    v = M.VolumeRender(R, storage="fp16")
    v.set_data(x)                                   # host floats, through the staging buffer
    np.testing.assert_array_equal(_bits(v.read(M.api.RES_DENSITY)), _bits(ref))
    v2 = M.VolumeRender(R, storage="fp16")
    v2.set_data(torch.from_numpy(x).cuda())         # device floats
    np.testing.assert_array_equal(_bits(v2.read(M.api.RES_DENSITY)), _bits(ref))
    # the grid takes half the bytes
    f = M.VolumeRender(R)
    assert f.info().device_bytes - v.info().device_bytes == 2 * R ** 3


def test_generated_grid_is_the_rounded_fp32_grid():
    import mrpnn_b200 as M
    M.init()
    R = 48
    f = M.VolumeRender(R)
    f.generate_fbm(5, 6.0)
    h = M.VolumeRender(R, storage="fp16")
    h.generate_fbm(5, 6.0)
    ref = f.read(M.api.RES_DENSITY).astype(np.float16).astype(np.float32)
    np.testing.assert_array_equal(_bits(h.read(M.api.RES_DENSITY)), _bits(ref))


def test_resources_identical(pair):
    import mrpnn_b200 as M
    h, f = pair
    assert _bits(np.float32(h.max_density)) == _bits(np.float32(f.max_density))
    for m in range(9):
        np.testing.assert_array_equal(_bits(h.read(M.api.RES_MIP, m)), _bits(f.read(M.api.RES_MIP, m)))
    np.testing.assert_array_equal(h.read(M.api.RES_OCCUPANCY), f.read(M.api.RES_OCCUPANCY))
    for v in (h, f):
        v.Update_TR(LIGHT, 64.0)
        v.Update_CachedTR(LIGHT, 64.0)
    for i in range(8):
        np.testing.assert_array_equal(_bits(h.read(M.api.RES_TR, i)), _bits(f.read(M.api.RES_TR, i)))
    np.testing.assert_array_equal(_bits(h.read(M.api.RES_BAKED_TR)), _bits(f.read(M.api.RES_BAKED_TR)))


def test_images_identical(pair):
    import mrpnn_b200 as M
    h, f = pair
    ori, up, right = view_frame()
    imgs = {}
    for name, v in (("fp16", h), ("fp32", f)):
        v.SetPrecision(M.FP32)
        pt = v.Render(48, ori, up, right, LIGHT, rt=M.VolumeRender.PT, alpha=64.0, multiScatter=64, sampleNum=1,
                      spp=4, seed=7)
        nn32 = v.Render(80, ori, up, right, LIGHT, rt=M.VolumeRender.MRPNN, alpha=64.0, sampleNum=1, seed=7)
        v.SetPrecision(M.BF16)
        nn16 = v.Render(80, ori, up, right, LIGHT, rt=M.VolumeRender.MRPNN, alpha=64.0, sampleNum=1, seed=7)
        v.SetPrecision(M.FP32)
        imgs[name] = (pt, nn32, nn16)
    for a, b in zip(imgs["fp16"], imgs["fp32"]):
        assert (a[..., 3] > 0).any()
        np.testing.assert_array_equal(_bits(a), _bits(b))


def test_batch_rays_identical(pair):
    import mrpnn_b200 as M
    h, f = pair
    rng = np.random.default_rng(9)
    n = 512
    ori = np.tile(np.asarray([0.75, 0.75, 0.75], np.float32), (n, 1))
    d = (-ori + rng.normal(0, 0.15, (n, 3))).astype(np.float32)
    outs = []
    for v in (h, f):
        pt = v.GetRadiances(ori, d, LIGHT, alpha=64.0, multiScatter=16, g=0.857, sampleNum=2)
        nn = v.GetRadiances(ori, d, LIGHT, alpha=64.0, g=0.857, rt=M.VolumeRender.MRPNN)
        tr = v.GetTrs(64.0, ori * 0.2, d, LIGHT, g=0.857, sampleNum=2, seed=3)
        outs.append((pt, nn, tr))
    for a, b in zip(*outs):
        np.testing.assert_array_equal(_bits(a), _bits(b))


def test_pyramid_from_a_larger_fp16_grid():
    """R > 512: the first pyramid step resamples the fp16 grid itself (to
    512^3) before the nine levels; compared on the device, no host copy of
    the grid."""
    import torch

    import mrpnn_b200 as M
    M.init()
    R = 600
    h = M.VolumeRender(R, storage="fp16")
    h.generate_fbm(2, 8.0)
    wide = torch.empty(R ** 3, dtype=torch.float32, device="cuda")
    M.api._check(M.api.lib().mrp_volume_read(h._h, M.api.RES_DENSITY, 0, C.c_void_p(wide.data_ptr()), None, 1))
    f = M.VolumeRender(R)
    f.set_data(wide)
    del wide
    for v in (h, f):
        v.Update()
    assert _bits(np.float32(h.max_density)) == _bits(np.float32(f.max_density))
    for m in range(9):
        np.testing.assert_array_equal(_bits(h.read(M.api.RES_MIP, m)), _bits(f.read(M.api.RES_MIP, m)))
    np.testing.assert_array_equal(h.read(M.api.RES_OCCUPANCY), f.read(M.api.RES_OCCUPANCY))
