"""The MRPNN predictor on the GPU against the CPU oracle (itself pinned to
the reference's own code by tests/test_oracle_pins.py).

Tolerances: first-hit decisions are exact (only +,-,*,/ and comparisons);
hit positions, features and the MLP differ only through the last bit of
log/exp/pow/atan/acos, so features agree to 1e-5 relative and the FP32 MLP
to the 1e-4 relative bound of the drop-in contract."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_scene import LIGHT, Scene, view_frame

pytestmark = pytest.mark.gpu

MLP_RTOL = 1e-4      # FP32 predictor vs the reference predictor, relative
MLP_ATOL = 1e-6      # floor for outputs at 0 (relu / exp(x)-1 near 0)


@pytest.fixture(scope="module")
def scene():
    return Scene(R=64)


def test_mlp_fp32_matches_reference_golden(golden):
    """GPU FP32 MLP vs RadiancePredictInternal compiled from the reference."""
    import mrpnn_b200 as M
    M.init()
    for tag in ("grey", "rgb"):
        out = M.predict_features(golden["mlp_feat"], golden["mlp_gamma"], 0.857, golden[f"mlp_sr_{tag}"])
        ref = golden[f"mlp_out_{tag}"]
        np.testing.assert_allclose(out, ref, rtol=MLP_RTOL, atol=MLP_ATOL)


def test_mlp_fp32_random_features():
    import mrpnn_b200 as M
    M.init()
    rng = np.random.default_rng(11)
    n = 1000
    feat = np.concatenate([rng.uniform(0, 1.5, (n, 192)), rng.uniform(0, 1, (n, 192)),
                           rng.uniform(0, 3, (n, 192))], 1).astype(np.float32)
    gam = rng.uniform(0, np.pi, n).astype(np.float32)
    for sr in ((1.0, 1.0, 1.0), (0.99, 0.9, 0.8), (0.9, 0.9, 0.7)):
        out = M.predict_features(feat, gam, 0.857, sr)
        ref = O.mlp_f32(feat, gam, 0.857, sr)
        np.testing.assert_allclose(out, ref, rtol=MLP_RTOL, atol=MLP_ATOL)


def test_mlp_fp32_device_buffers():
    import torch
    import mrpnn_b200 as M
    M.init()
    rng = np.random.default_rng(12)
    feat = rng.uniform(0, 1.5, (300, 576)).astype(np.float32)
    gam = rng.uniform(0, 3, 300).astype(np.float32)
    out = M.predict_features(torch.from_numpy(feat).cuda(), torch.from_numpy(gam).cuda(), 0.5, (1, 1, 1))
    ref = O.mlp_f32(feat, gam, 0.5, (1, 1, 1))
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=MLP_RTOL, atol=MLP_ATOL)


def test_first_hit(scene):
    rng = np.random.default_rng(1)
    n = 4096
    ori = (np.array([0.75, 0.75, 0.75]) + rng.normal(0, 0.05, (n, 3))).astype(np.float32)
    d = (-ori + rng.normal(0, 0.25, (n, 3))).astype(np.float32)
    got = scene.vol.first_hit(ori, d, scene.alpha)
    L = O.lib()
    ref = np.zeros((n, 4), np.float32)
    h = np.zeros(3, np.float32)
    for i in range(n):
        ref[i, 3] = L.orc_first_hit(C.byref(scene.orc.c), ori[i], d[i], scene.alpha, h)
        ref[i, :3] = h
    np.testing.assert_array_equal(got[:, 3], ref[:, 3])
    assert ref[:, 3].sum() > n // 4
    np.testing.assert_allclose(got[:, :3], ref[:, :3], rtol=0, atol=2e-6)
    assert np.mean(np.all(got == ref, axis=1)) > 0.9   # most hits are bit-identical


def test_gather(scene):
    rng = np.random.default_rng(2)
    n = 256
    pos = rng.uniform(-0.45, 0.45, (n, 3)).astype(np.float32)
    bases = np.zeros((n, 12), np.float32)
    L = O.lib()
    for i in range(n):
        cur = C.c_uint32(0)
        m9 = np.zeros(9, np.float32)
        l9 = np.zeros(9, np.float32)
        L.orc_basis(rng.normal(size=3).astype(np.float32), 0.1, i, 0, 0, 0, C.byref(cur), m9)
        cur = C.c_uint32(0)
        L.orc_basis(LIGHT, 0.1, i, 1, 0, 0, C.byref(cur), l9)
        bases[i, :9], bases[i, 9:] = m9, l9[:3]
    feat, gam = scene.vol.gather_features(pos, bases, LIGHT, scene.g, scene.alpha)
    ref = np.zeros((n, 576), np.float32)
    rg = np.zeros(n, np.float32)
    f = np.zeros(576, np.float32)
    gm = np.zeros(1, np.float32)
    for i in range(n):
        b = bases[i]
        L.orc_setup_input(C.byref(scene.orc.c), 1, pos[i], b[0:3].copy(), b[3:6].copy(), b[6:9].copy(),
                          b[9:12].copy(), LIGHT, scene.g, scene.alpha, f, gm)
        ref[i], rg[i] = f, gm[0]
    np.testing.assert_allclose(feat, ref, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(gam, rg, rtol=0, atol=2e-5)


def _render_pair(scene, W, frame=0, launches=1, sr=0.99):
    import mrpnn_b200 as M
    ori, up, right = view_frame()
    out = scene.vol.Render((W, W), ori, up, right, LIGHT, M.VolumeRender.MRPNN, scene.g, scene.alpha,
                           sampleNum=launches, seed=3)
    acc = np.zeros((W * W, 4), np.float32)
    for k in range(launches):
        view = O.make_view(W, W, ori, up, right, LIGHT, alpha=scene.alpha, g=scene.g, seed=3, frame=frame + k)
        res = O.predict_pixels(scene.orc, view, np.arange(W * W, dtype=np.int32))
        rate = np.float32(1.0) / np.float32(1 + k)
        acc = acc * (np.float32(1) - rate) + res * rate
    return out.reshape(-1, 4), acc


def test_predict_render_one_launch(scene):
    got, ref = _render_pair(scene, 64)
    assert np.array_equal(got[:, 3] > 0, ref[:, 3] > 0)      # same pixels hit
    assert (ref[:, 3] > 0).sum() > 500
    ok = np.isclose(got, ref, rtol=MLP_RTOL, atol=MLP_ATOL).all(axis=1)
    assert ok.mean() > 0.999, np.argwhere(~ok)[:5]


def test_predict_render_running_mean(scene):
    got, ref = _render_pair(scene, 32, launches=3)
    np.testing.assert_allclose(got, ref, rtol=MLP_RTOL, atol=MLP_ATOL)


def test_predict_intermediates(scene):
    """Hit points, bases, gamma and features inside the render kernel against
    the oracle's NNPredict, pixel by pixel."""
    import mrpnn_b200 as M
    W = 32
    ori, up, right = view_frame()
    view = scene.vol.make_view((W, W), ori, up, right, LIGHT, scene.g, scene.alpha, seed=3)
    rgba, aux, feat = scene.vol.predict_debug(view)
    oview = O.make_view(W, W, ori, up, right, LIGHT, alpha=scene.alpha, g=scene.g, seed=3, frame=0)
    r_rgba, r_feat, r_gamma, r_hit = O.predict_pixels(scene.orc, oview, np.arange(W * W, dtype=np.int32),
                                                      want_features=True)
    L = O.lib()
    hit = r_hit[:, 3] > 0
    np.testing.assert_array_equal(aux[:, 3], r_hit[:, 3])
    np.testing.assert_allclose(aux[hit, :3], r_hit[hit, :3], rtol=0, atol=2e-6)
    # bases from the pixel stream (draws 0.. after InitRand)
    bases = np.zeros((W * W, 12), np.float32)
    for p in range(W * W):
        d0 = np.zeros(3, np.float32)
        L.orc_camera_ray(C.byref(oview), p // W, p % W, d0)
        d = d0 / np.float32(np.sqrt(np.float32(np.dot(d0, d0))))
        cur = C.c_uint32(0)
        m9 = np.zeros(9, np.float32)
        l9 = np.zeros(9, np.float32)
        L.orc_basis(d.astype(np.float32), 0.1, p, 0, 0, 3, C.byref(cur), m9)
        L.orc_basis(LIGHT, 0.1, p, 0, 0, 3, C.byref(cur), l9)
        bases[p, :9], bases[p, 9:] = m9, l9[:3]
    np.testing.assert_allclose(aux[hit, 5:17], bases[hit], rtol=0, atol=1e-5, err_msg="bases")
    np.testing.assert_allclose(aux[hit, 4], r_gamma[hit], rtol=0, atol=2e-5, err_msg="gamma")
    np.testing.assert_allclose(feat[hit], r_feat[hit], rtol=1e-5, atol=1e-6, err_msg="features")
    np.testing.assert_allclose(rgba, r_rgba, rtol=MLP_RTOL, atol=MLP_ATOL, err_msg="rgba")


@pytest.mark.parametrize("case", ["empty", "corner", "full_face", "sdf"])
def test_first_hit_empty_space_replay(case):
    """The march replays its steps in front of the box of nonzero voxels as
    additions alone and drops rays that never reach it; the hits must stay
    those of the oracle's full march: an all-zero grid, one dense corner
    block, density touching a face of the grid, and negative (SDF) values."""
    import mrpnn_b200 as M
    M.init()
    R = 48
    grid = np.zeros((R, R, R), np.float32)
    if case == "corner":
        grid[R - 6:, R - 6:, R - 6:] = 1.0
    elif case == "full_face":
        grid[:, :, 0:5] = 0.8
    elif case == "sdf":
        grid[10:30, 12:30, 14:30] = -0.02
        grid[18:22, 18:22, 18:22] = 1.0
    vol = M.VolumeRender(R)
    vol.set_data(grid)
    vol.Update()
    alpha = 64.0
    rng = np.random.default_rng(7)
    n = 3000
    ori = (np.array([0.75, 0.75, 0.75]) + rng.normal(0, 0.1, (n, 3))).astype(np.float32)
    d = (-ori + rng.normal(0, 0.3, (n, 3))).astype(np.float32)
    got = vol.first_hit(ori, d, alpha)
    sc = O.SceneBuf(vol.read(M.api.RES_DENSITY), R, vol.max_density)
    L = O.lib()
    ref = np.zeros((n, 4), np.float32)
    h = np.zeros(3, np.float32)
    for i in range(n):
        ref[i, 3] = L.orc_first_hit(C.byref(sc.c), ori[i], d[i], alpha, h)
        ref[i, :3] = h
    np.testing.assert_array_equal(got[:, 3], ref[:, 3])
    if case == "empty":
        assert ref[:, 3].sum() == 0
    else:
        assert ref[:, 3].sum() > 0
    np.testing.assert_allclose(got[:, :3], ref[:, :3], rtol=0, atol=2e-6)


# The texture unit's filter weights are 1/256 steps (a weight is off by at
# most 1/512): per trilinear fetch the value moves by at most 3/512 of the
# footprint's range, per bilinear LUT fetch by 2/512 of its range.  The
# features of the hardware-filtered gather are held to the oracle's exact
# features at these bounds (absolute, in feature units), with the bulk far
# inside them.
HW_FEAT_MAX_ABS = 0.05
HW_FEAT_P99_ABS = 5e-3


@pytest.mark.parametrize("hw", [False, True], ids=["software", "texture"])
@pytest.mark.parametrize("prec", ["BF16", "FP8"])
def test_fp16_features(scene, prec, hw):
    """The tensor-core forms' stencil features -- fp16, the hardware log2 and
    the per-point LUT factor of X_Hg -- against the oracle's exact features,
    and the debug launch's image against mrp_render's image of the same
    launch.  Software filters (gather_filter 0): within fp16 rounding (2^-11
    relative).  The texture unit's filters (gather_filter 1, the default, as
    the reference's tex3D / tex2D): within the weight quantisation's bound."""
    import mrpnn_b200 as M
    W = 48
    ori, up, right = view_frame()
    view = scene.vol.make_view((W, W), ori, up, right, LIGHT, scene.g, scene.alpha, seed=3)
    scene.vol.SetPrecision(getattr(M, prec))
    scene.vol.SetGatherFilter(hw)
    try:
        rgba, aux, feat = scene.vol.predict_debug(view)
        img = np.empty((W, W, 4), np.float32)
        scene.vol.render_view(view, M.VolumeRender.MRPNN, 1, img)
    finally:
        scene.vol.SetPrecision(M.FP32)
        scene.vol.SetGatherFilter(True)
    oview = O.make_view(W, W, ori, up, right, LIGHT, alpha=scene.alpha, g=scene.g, seed=3, frame=0)
    _, r_feat, _, r_hit = O.predict_pixels(scene.orc, oview, np.arange(W * W, dtype=np.int32), want_features=True)
    hit = r_hit[:, 3] > 0
    assert hit.sum() > 100
    np.testing.assert_array_equal(aux[:, 3], r_hit[:, 3])
    if not hw:
        np.testing.assert_allclose(feat[hit], r_feat[hit], rtol=2e-3, atol=2e-5)
    else:
        err = np.abs(feat[hit] - r_feat[hit])
        print(f"texture gather: max |err| {err.max():.2e}, p99 {np.percentile(err, 99):.2e}, "
              f"p50 {np.median(err):.2e}; per channel max {err.reshape(-1, 3, 192).max(axis=(0, 2))}")
        assert err.max() < HW_FEAT_MAX_ABS
        assert np.percentile(err, 99) < HW_FEAT_P99_ABS
        # the filter is the texture unit's: some features differ from the
        # software filter's beyond fp16 rounding
        assert (err > 2e-3 * np.abs(r_feat[hit]) + 2e-5).any()
    np.testing.assert_array_equal(rgba.reshape(W, W, 4), img)


def test_texture_gather_follows_updates():
    """The texture copies of the BF16 gather are refreshed whenever a builder
    rewrites the linear levels: after a change of light (TR levels), of g (the
    LUT) and of the volume's data (pyramid), a render equals the render of a
    fresh volume that never saw the earlier state, bit for bit."""
    import mrpnn_b200 as M
    M.init()
    ori, up, right = view_frame()
    W = 64
    L2 = np.array([-0.5, 0.7, 0.2], np.float32)
    L2 = (L2 / np.float32(np.linalg.norm(L2))).astype(np.float32)

    def fresh(seed, L, g):
        v = M.VolumeRender(64)
        v.generate_fbm(seed, 4.0)
        v.Update()
        v.SetScatterRate(0.99)
        v.SetSky(0.05)
        v.SetPrecision(M.BF16)
        return v, v.Render((W, W), ori, up, right, L, M.VolumeRender.MRPNN, g, 64.0, sampleNum=1, seed=5)

    v, first = fresh(0, LIGHT, 0.857)
    for seed, L, g in ((0, L2, 0.857), (0, L2, 0.5), (7, L2, 0.5)):
        if seed != 0:
            v.generate_fbm(seed, 4.0)
            v.Update()
        got = v.Render((W, W), ori, up, right, L, M.VolumeRender.MRPNN, g, 64.0, sampleNum=1, seed=5)
        _, want = fresh(seed, L, g)
        assert (want[..., 3] > 0).sum() > 100
        np.testing.assert_array_equal(got, want)
    assert not np.array_equal(first, got)

