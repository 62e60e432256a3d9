"""Batch ray APIs (GetRadiances / GetSamples / GetTrs, core/volume.cu:405-479,
710-834) on the GPU against the oracle's restatements, same Philox streams.

Stochastic results agree until a transcendental's last bit flips an
accept/reject decision, so they are compared as in the tracer test: most
tasks reproduce to float rounding, and the mean over tasks agrees within a
few standard errors.  GetRadiances in MRPNN mode on a view's own camera rays
must equal the rendered frame exactly (same hit, same basis stream)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_scene import LIGHT, Scene, view_frame

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    return Scene(R=64)


def _close_fraction(a, b):
    return float(np.mean(np.isclose(a, b, rtol=1e-5, atol=1e-7).all(axis=1)))


def _inside_points(n, rng):
    return rng.uniform(-0.3, 0.3, (n, 3)).astype(np.float32)


def _unit(n, rng):
    d = rng.normal(size=(n, 3))
    return (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)


def test_get_samples_matches_oracle(scene):
    rng = np.random.default_rng(5)
    n, spp = 512, 8
    ori, dirs = _inside_points(n, rng), _unit(n, rng)
    ldir = _unit(n, rng)
    alpha = rng.uniform(16, 96, n).astype(np.float32)
    g = rng.uniform(0.2, 0.9, n).astype(np.float32)
    sc = rng.uniform(0.8, 0.99, n).astype(np.float32)
    got = scene.vol.GetSamples(alpha, ori, dirs, ldir, g, sc, (1, 1, 1), multiScatter=32, sampleNum=spp, seed=3)
    ref = O.get_samples(scene.orc, alpha, ori, dirs, ldir, g, sc, (1, 1, 1), 32, spp, 3)
    assert _close_fraction(got, ref) > 0.8
    assert abs(got.mean() - ref.mean()) < 0.03 * ref.mean()


def test_get_trs_matches_oracle(scene):
    rng = np.random.default_rng(6)
    n = 1024
    ori, dirs = _inside_points(n, rng), _unit(n, rng)
    got = scene.vol.GetTrs(64.0, ori, dirs, LIGHT, (1.0, 0.9, 0.8), g=0.857, sampleNum=16, seed=9)
    ref = O.get_trs(scene.orc, 64.0, ori, dirs, LIGHT, (1.0, 0.9, 0.8), 0.857, 16, 9)
    assert _close_fraction(got, ref) > 0.8
    assert abs(got.mean() - ref.mean()) < 0.02 * ref.mean()


def test_get_radiances_pt_matches_oracle(scene):
    import mrpnn_b200 as M
    rng = np.random.default_rng(7)
    n, spp = 400, 32
    dirs = _unit(n, rng)
    ori = (-dirs * 1.5 + rng.uniform(-0.2, 0.2, (n, 3))).astype(np.float32)
    scene.vol.SetNeeMode(True)
    try:
        got = scene.vol.GetRadiances(ori, dirs, LIGHT, (1, 1, 1), scene.alpha, 64, scene.g, spp, M.VolumeRender.PT)
    finally:
        scene.vol.SetNeeMode(False)
    view = O.make_view(n, 1, (0, 0, 0), (0, 1, 0), (1, 0, 0), LIGHT, alpha=scene.alpha, g=scene.g,
                       multi_scatter=64, spp=spp, seed=0, frame=0)
    s, s2 = O.trace_rays(scene.orc, view, ori, dirs)
    mean = s / spp
    var = np.maximum(s2 / spp - mean ** 2, 0) * spp / (spp - 1)
    z = (got - mean) / (np.sqrt(2 * var / spp) + 1e-7)
    assert np.mean(np.abs(z) < 4) >= 0.995
    assert _close_fraction(got, mean.astype(np.float32)) > 0.5


def test_get_radiances_mrpnn_equals_frame(scene):
    import mrpnn_b200 as M
    W = 32
    ori, up, right = view_frame()
    frame = scene.vol.Render((W, W), ori, up, right, LIGHT, M.VolumeRender.MRPNN, scene.g, scene.alpha,
                             sampleNum=1, seed=0).reshape(-1, 4)
    view = O.make_view(W, W, ori, up, right, LIGHT, alpha=scene.alpha, g=scene.g, seed=0, frame=0)
    dirs = np.empty((W * W, 3), np.float32)
    d = np.empty(3, np.float32)
    for p in range(W * W):
        O.lib().orc_camera_ray(C.byref(view), p // W, p % W, d)
        dirs[p] = d
    oris = np.broadcast_to(np.asarray(ori, np.float32), (W * W, 3))
    got = scene.vol.GetRadiances(oris, dirs, LIGHT, (1, 1, 1), scene.alpha, 1, scene.g, 1, M.VolumeRender.MRPNN)
    np.testing.assert_allclose(got, frame[:, :3], rtol=1e-5, atol=1e-6)


def test_gather_tiles_matches_oracle(scene):
    """GatherData (773 tile features) on the GPU against the oracle, itself
    pinned bit for bit to the reference's NNGatherSamples: the depth marches
    use only +, -, *, /, sqrt, so only the last bits of log / acos / exp may
    differ."""
    TW = 12
    ori, up, right = view_frame()
    got = scene.vol.GatherData((TW, TW), ori, up, right, LIGHT, alpha=scene.alpha, g=scene.g, pixelOffset=(3, 5),
                               seed=5, frame=2)
    view = O.make_view(TW, TW, ori, up, right, LIGHT, alpha=scene.alpha, g=scene.g, seed=5, frame=2)
    ref = O.gather_tiles(scene.orc, view, 3, 5)
    assert (ref[:, 0] != -1000).sum() > 40
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-5)
