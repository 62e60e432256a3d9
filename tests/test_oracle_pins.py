"""The CPU oracle against the reference's own render code.

Golden vectors in tests/golden/ref_pins.npz come from the reference's
core/vector.cu, core/radiancePredict.cu, core/renderResources.cu and
core/render.cuh compiled on the CPU (tests/golden/make_golden.py).  Every
case here is bit-exact: the oracle keeps the reference's float rounding order.
"""
import ctypes as C
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden.make_golden import SCENE, build_scene, camera, light_dir


def test_mlp_matches_reference(oracle, golden):
    feat, gam = golden["mlp_feat"], golden["mlp_gamma"]
    for tag in ("grey", "rgb"):
        out = oracle.mlp_f32(feat, gam, 0.857, golden[f"mlp_sr_{tag}"])
        np.testing.assert_array_equal(out, golden[f"mlp_out_{tag}"])


def test_mlp_f64_close_to_f32(oracle, golden):
    feat, gam = golden["mlp_feat"], golden["mlp_gamma"]
    a = oracle.mlp_f32(feat, gam, 0.857, golden["mlp_sr_rgb"])
    d = oracle.mlp_f64(feat, gam, 0.857, golden["mlp_sr_rgb"])
    rel = np.abs(a - d) / np.maximum(np.abs(d), 1e-6)
    assert rel.max() < 1e-4


def test_stencil_tables(oracle, golden):
    off, layer, typ, li, _ = oracle.stencil_tables()
    np.testing.assert_array_equal(off, golden["st_offset"])
    np.testing.assert_array_equal(layer, (golden["st_layer"] + np.float32(0.1)).astype(np.int32))
    np.testing.assert_array_equal(typ, golden["st_type"])
    np.testing.assert_array_equal(li, golden["st_localindex"])
    data = C.POINTER(C.c_float)()
    cnt = C.c_int()
    assert oracle.lib().orc_model_tensor(b"STENCIL_DIRS", C.byref(data), C.byref(cnt)) == 0
    dirs = np.ctypeslib.as_array(data, (cnt.value,)).reshape(160, 3)
    np.testing.assert_array_equal(dirs, golden["st_dirs"][:160])


def test_maths(oracle, golden):
    L = oracle.lib()
    hg = np.array([L.orc_hg(c, g) for c, g in golden["hg_in"]], np.float32)
    np.testing.assert_array_equal(hg, golden["hg_out"])
    out = np.zeros(3, np.float32)
    for i in range(len(golden["shg_e"])):
        e = golden["shg_e"][i]
        L.orc_sample_hg(e[0], e[1], np.ascontiguousarray(golden["shg_v"][i]), golden["shg_g"][i], out)
        np.testing.assert_array_equal(out, golden["shg_out"][i])
    p, d = golden["rb_p"], golden["rb_d"]
    off = np.array([L.orc_ray_box_offset(p[i], d[i]) for i in range(len(p))], np.float32)
    dist = np.array([L.orc_ray_box_distance(p[i], d[i]) for i in range(len(p))], np.float32)
    np.testing.assert_array_equal(off, golden["rb_off"])
    np.testing.assert_array_equal(dist, golden["rb_dist"])


@pytest.fixture(scope="module")
def scene(oracle):
    return build_scene()


def test_scene_is_reproducible(scene, golden):
    d = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    assert d(scene.mips) == str(golden["scene_digest_mips"])
    assert d(scene.tr) == str(golden["scene_digest_tr"])
    assert d(scene.lut) == str(golden["scene_digest_lut"])


def test_first_hit(oracle, scene, golden):
    L = oracle.lib()
    h = np.zeros(3, np.float32)
    for o, d, ref in zip(golden["fh_ori"], golden["fh_dir"], golden["fh_out"]):
        a = L.orc_first_hit(C.byref(scene.c), o, d, SCENE["alpha"], h)
        assert a == int(ref[3])
        np.testing.assert_array_equal(h, ref[:3])


def test_basis(oracle, golden):
    L = oracle.lib()
    for i, (v, ref) in enumerate(zip(golden["basis_v"], golden["basis_out"])):
        cur = C.c_uint32(0)
        o9 = np.zeros(9, np.float32)
        L.orc_basis(np.ascontiguousarray(v), 0.1, i, 0, 3, 11, C.byref(cur), o9)
        np.testing.assert_array_equal(o9, ref)


def test_setup_input(oracle, scene, golden):
    L = oracle.lib()
    Ld = light_dir()
    f = np.zeros(576, np.float32)
    gm = np.zeros(1, np.float32)
    for p, b, ref_f, ref_g in zip(golden["si_pos"], golden["si_bases"], golden["si_feat"], golden["si_gamma"]):
        b = np.ascontiguousarray(b)
        L.orc_setup_input(C.byref(scene.c), 1, p, b[0:3].copy(), b[3:6].copy(), b[6:9].copy(), b[9:12].copy(), Ld,
                          SCENE["g"], SCENE["alpha"], f, gm)
        np.testing.assert_array_equal(f, ref_f)
        assert gm[0] == ref_g


def test_predict_pixels(oracle, scene, golden):
    W = 16
    ori, up, right = camera(W)
    view = oracle.make_view(W, W, ori, up, right, light_dir(), alpha=SCENE["alpha"], g=SCENE["g"], seed=5, frame=2)
    rgba = oracle.predict_pixels(scene, view, np.arange(W * W, dtype=np.int32))
    np.testing.assert_array_equal(rgba, golden["pp_rgba"])
    assert (rgba[:, 3] > 0).sum() > 50   # the view actually hits the cloud


def test_trace_samples(oracle, scene, golden):
    W = 16
    ori, up, right = camera(W)
    for (pix, k), ref in zip(golden["ts_cases"], golden["ts_out"]):
        view = oracle.make_view(W, W, ori, up, right, light_dir(), alpha=SCENE["alpha"], g=SCENE["g"],
                                multi_scatter=64, spp=int(k) + 1, seed=5, frame=2)
        _, s, _ = oracle.trace_pixels(scene, view, np.array([pix], np.int32))
        if k > 0:
            view.spp = int(k)
            _, s0, _ = oracle.trace_pixels(scene, view, np.array([pix], np.int32))
            s = s - s0
        np.testing.assert_array_equal(s[0].astype(np.float32), ref[:3])


def test_transmittance(oracle, scene, golden):
    L = oracle.lib()
    Ld = light_dir()
    for i, (p, ref) in enumerate(zip(golden["tr_pos"], golden["tr_out"])):
        dis = L.orc_ray_box_distance(p, Ld)
        v = L.orc_tr(C.byref(scene.c), p, Ld, dis, SCENE["alpha"], i, 0, 0, 9, 2)
        assert np.float32(v) == ref


def test_philox_known_answers(oracle):
    """Philox-4x32-10 known-answer vectors of the Random123 distribution."""
    L = oracle.lib()
    out = np.zeros(4, np.uint32)
    cases = [
        ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
        ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
        ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
         [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
    ]
    for c, k, want in cases:
        L.orc_philox4x32_10(np.array(c, np.uint32), np.array(k, np.uint32), out)
        assert list(out) == want


@pytest.mark.skipif(not O.ref_available(), reason="reference checker not available")
def test_live_reference_mlp_small(oracle):
    """Re-run the reference MLP (live build) on fresh random features."""
    rng = np.random.default_rng(7)
    feat = rng.uniform(0, 2.0, (32, 576)).astype(np.float32)
    gam = rng.uniform(0, np.pi, 32).astype(np.float32)
    np.testing.assert_array_equal(oracle.mlp_f32(feat, gam, 0.6, (0.95, 0.95, 0.95)),
                                  oracle.ref_mlp(feat, gam, 0.6, (0.95, 0.95, 0.95)))


def test_gather_tiles(oracle, scene, golden):
    """GatherData / NNGatherSamples (773 floats per tile) against the
    reference's own code; tile 0 carries the kernel's debug multiplies."""
    TW = 6
    ori, up, right = camera(TW)
    view = oracle.make_view(TW, TW, ori, up, right, light_dir(), alpha=SCENE["alpha"], g=SCENE["g"], seed=5, frame=2)
    got = oracle.gather_tiles(scene, view, 3, 5)
    ref = golden["tile_out"]
    np.testing.assert_array_equal(got, ref)
    assert (ref[:, 0] != -1000).sum() > 20     # most tiles see the cloud


# ---------------------------------------------------------------------------
# volume builders, pinned to core/volume.cu compiled on the CPU
# ---------------------------------------------------------------------------
from tests.golden.make_golden import BAKE_RES, LUT_GS, digest, lut_queries, smooth_lut  # noqa: E402


def test_pyramid_matches_reference(oracle, golden):
    """VolumeRender::Update's CPU pyramid (core/volume.cu:835-882, 1474-1515),
    the 32^3 scene and a 300^3 grid (non power of two)."""
    R = SCENE["R"]
    vol = oracle.fbm_volume(R, SCENE["seed"], SCENE["freq"])
    assert digest(oracle.build_pyramid(vol, R)) == str(golden["vol_pyramid_digest"])
    v300 = oracle.fbm_volume(300, 3, 5.0)
    assert digest(oracle.build_pyramid(v300, 300)) == str(golden["vol_pyramid300_digest"])


def test_tr_levels_match_reference(oracle, golden):
    """Update_TR: Fill_TR over the mip textures (the device branch) and
    Sample_TR (the host branch) give the same levels, and the oracle's."""
    R = SCENE["R"]
    vol = oracle.fbm_volume(R, SCENE["seed"], SCENE["freq"])
    tr = oracle.tr_mips(oracle.build_pyramid(vol, R), SCENE["alpha"], light_dir())
    assert digest(tr) == str(golden["vol_tr_digest"])
    assert str(golden["vol_tr_cpu_digest"]) == str(golden["vol_tr_digest"])


def test_hg_lut_texels_match_reference(oracle, golden):
    """Fill_Hg (core/volume.cu:1322-1400) with the reference's digit
    permutations at the same per-texel shift bn: bit for bit."""
    tex = golden["vol_lut_texels"]
    for tag, g in LUT_GS:
        np.testing.assert_array_equal(oracle.hg_lut_texels(g, SCENE["lut_seed"], tex), golden[f"vol_lut_{tag}"])


def test_get_hg_lut_matches_reference(golden):
    """VolumeRender::GetHGLut (core/volume.cu:1424-1442) through the
    library's host-only mrp_hg_lut_lookup."""
    import mrpnn_b200 as M
    lut = smooth_lut()
    got = np.array([M.hg_lut_lookup(lut, c, a) for c, a in golden["vol_getlut_q"]], np.float32)
    np.testing.assert_array_equal(got, golden["vol_getlut_out"])


def test_baked_tr_matches_reference(oracle, golden):
    """Fill_BakeTR (core/volume.cu:1562-1587) per voxel, the estimates'
    streams restarted as the kernel's InitRand does."""
    R = SCENE["R"]
    vol = oracle.fbm_volume(R, SCENE["seed"], SCENE["freq"])
    md = oracle.lib().orc_max_density(vol, vol.size)
    sc = oracle.SceneBuf(vol, R, md)
    got = oracle.baked_tr_voxels(sc, SCENE["alpha"], light_dir(), BAKE_RES, SCENE["lut_seed"], golden["vol_bake_vox"])
    np.testing.assert_array_equal(got, golden["vol_bake_out"])


def test_halton_permutations_are_the_references():
    """The model file carries the first 28 entries of the reference's
    RadicalInversePermutations_ (bases 2, 3, 5, 7, 11)."""
    from oracle import oracle as O
    O.lib()
    data = C.POINTER(C.c_float)()
    cnt = C.c_int()
    assert O.lib().orc_model_tensor(b"HALTON_PERMS", C.byref(data), C.byref(cnt)) == 0
    perms = np.ctypeslib.as_array(data, (cnt.value,)).astype(int)
    assert list(perms[:2]) == [0, 1] and sorted(perms[17:28]) == list(range(11))
    assert list(perms) == [0, 1, 2, 1, 0, 4, 1, 2, 3, 0, 6, 2, 4, 1, 0, 5, 3, 8, 3, 5, 4, 7, 2, 6, 9, 1, 10, 0]


@pytest.mark.skipif(not O.ref_available(), reason="reference checker not available")
def test_live_reference_volume_builders(oracle):
    """The volume builders re-run live on inputs the golden file does not
    hold: a 40^3 grid, another light, another g and bake resolution."""
    R = 40
    vol = oracle.fbm_volume(R, 9, 3.0)
    mips = oracle.build_pyramid(vol, R)
    np.testing.assert_array_equal(mips, oracle.ref_pyramid(vol, R))
    L = np.array([-0.6, 0.7, 0.38], np.float32)
    L /= np.float32(np.sqrt(np.float32(np.dot(L, L))))
    np.testing.assert_array_equal(oracle.tr_mips(mips, 23.0, L), oracle.ref_tr(vol, R, 23.0, L))
    tex = np.random.default_rng(4).choice(512 * 512, 64, replace=False).astype(np.int32)
    np.testing.assert_array_equal(oracle.hg_lut_texels(0.3, 11, tex), oracle.ref_hg_texels(0.3, 11, tex))
    md = oracle.lib().orc_max_density(vol, vol.size)
    vox = np.random.default_rng(5).choice(32 ** 3, 200, replace=False).astype(np.int64)
    sc = oracle.SceneBuf(vol, R, md)
    np.testing.assert_array_equal(oracle.baked_tr_voxels(sc, 23.0, L, 32, 3, vox),
                                  oracle.ref_bake_voxels(vol, R, md, 23.0, L, 32, 3, vox))


# ---------------------------------------------------------------------------
# environment map: SetHDRI's equirect texture sampled by SkyBox
# ---------------------------------------------------------------------------
from tests.golden.make_golden import HDRI_ENV_EXP, smooth_hdri  # noqa: E402


@pytest.fixture(scope="module")
def hdri_scene(oracle, scene):
    return oracle.SceneBuf(scene.density, scene.res, scene.max_density, scene.mips, scene.tr, scene.lut,
                           baked=scene.baked, baked_res=scene.baked_res, scatter_rate=SCENE["sr"], sky=SCENE["sky"],
                           hdri=smooth_hdri(), env_exp=HDRI_ENV_EXP)


def _wide_camera(W):
    ori, up, right = camera(W)
    return ori, (up * np.float32(2.5)).astype(np.float32), (right * np.float32(2.5)).astype(np.float32)


def test_hdri_predict_pixels(oracle, hdri_scene, golden):
    """NNPredict<MRPNN> returns SkyBox(dir) for the rays that miss the cloud."""
    W = 16
    ori, up, right = _wide_camera(W)
    view = oracle.make_view(W, W, ori, up, right, light_dir(), alpha=SCENE["alpha"], g=SCENE["g"], seed=5, frame=2)
    rgba = oracle.predict_pixels(hdri_scene, view, np.arange(W * W, dtype=np.int32))
    np.testing.assert_array_equal(rgba, golden["hdri_pp_rgba"])
    miss = rgba[:, 3] == 0
    assert miss.sum() > 100 and (~miss).sum() > 10
    assert np.ptp(rgba[miss, 0]) > 0.3          # the map varies across the missed pixels


def test_hdri_trace_samples(oracle, hdri_scene, golden):
    """CalculateRadiance: escaping paths add SkyBox(direction) x throughput."""
    W = 16
    ori, up, right = _wide_camera(W)
    for (pix, k), ref in zip(golden["hdri_ts_cases"], golden["hdri_ts_out"]):
        view = oracle.make_view(W, W, ori, up, right, light_dir(), alpha=SCENE["alpha"], g=SCENE["g"],
                                multi_scatter=64, spp=int(k) + 1, seed=5, frame=2)
        _, s, _ = oracle.trace_pixels(hdri_scene, view, np.array([pix], np.int32))
        if k > 0:
            view.spp = int(k)
            _, s0, _ = oracle.trace_pixels(hdri_scene, view, np.array([pix], np.int32))
            s = s - s0
        np.testing.assert_array_equal(s[0].astype(np.float32), ref[:3])


@pytest.mark.skipif(not O.ref_available(), reason="reference checker not available")
def test_env_light_pieces_match_reference(oracle):
    """Render's light choice with a map (core/volume.cu:494-509) is built from
    Roberts2, UniformSampleSphere and Image_host::Sample: each bit for bit."""
    L = oracle.lib()
    a, b = np.zeros(3, np.float32), np.zeros(3, np.float32)
    for n in (0, 1, 2, 7, 100, 12345):
        L.orc_roberts2(n, a)
        oracle.ref_volume().ref_vol_roberts2(n, b)
        np.testing.assert_array_equal(a, b)
    rng = np.random.default_rng(8)
    for ex, ey in rng.uniform(0, 1, (64, 2)).astype(np.float32):
        L.orc_uniform_sample_sphere(ex, ey, a)
        oracle.ref_volume().ref_vol_uniform_sample_sphere(ex, ey, b)
        np.testing.assert_array_equal(a, b)
    m = smooth_hdri()
    flat = np.ascontiguousarray(m).ravel()
    for u, v in rng.uniform(-0.05, 1.05, (64, 2)).astype(np.float32):
        L.orc_image_sample(flat, m.shape[1], m.shape[0], u, v, a)
        oracle.ref_volume().ref_vol_image_sample(flat, m.shape[1], m.shape[0], u, v, b)
        np.testing.assert_array_equal(a, b)


# ---------------------------------------------------------------------------
# the viewer frame (core/volume.cu:57-150, 285-372; core/ACES.cuh)
# ---------------------------------------------------------------------------
from tests.golden.make_golden import FINISH_MODES, VIEWER  # noqa: E402


def test_viewer_frame_matches_reference(oracle, scene, golden):
    """Two checkerboard PT frames with the running mean and the radiance
    histograms, then the finishing pass in every mode: bit for bit."""
    V = VIEWER
    W, H = V["W"], V["H"]
    ori, up, right = camera(W)
    tgt = golden["vw_target0"].reshape(H, W, 3)
    his = golden["vw_histo0"].reshape(H, W, 33)
    for fnum in (0, 1):
        view = oracle.make_view(W, H, ori, up, right, light_dir(), alpha=SCENE["alpha"], g=SCENE["g"],
                                multi_scatter=V["multi"], seed=V["seed"], frame=V["frame"] + fnum)
        tgt, his = oracle.frame_pt(scene, view, fnum, 1, 1, tgt, his)
    np.testing.assert_array_equal(tgt.ravel(), golden["vw_target"])
    np.testing.assert_array_equal(his.ravel(), golden["vw_histo"])
    for k, (pred, den, tone) in enumerate(FINISH_MODES):
        for fn in (0, 5):
            o8, h = oracle.frame_finish(tgt, his, fn, 1, pred, den, V["exposure"], tone)
            np.testing.assert_array_equal(o8.ravel(), golden[f"vw_rgba8_{k}_{fn}"])
            np.testing.assert_array_equal(h.ravel(), golden[f"vw_histo_{k}_{fn}"])
