"""The viewer frame (VolumeRender::Render(float3*, Histogram*, ...)) on the
GPU against the oracle: each frame's running mean and histograms from the
same starting state (paths agree until a transcendental's last bit flips a
decision), and the Denoise / tone / RGBA8 pass on the GPU's own buffers
(8-bit channels within 1: pow's last bit)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_scene import LIGHT, Scene, view_frame

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    return Scene(R=64, bake_res=64)


def _channels(img):
    return np.stack([(img >> s) & 0xFF for s in (16, 8, 0)], -1).astype(np.int32)


@pytest.mark.parametrize("checker,denoise,tone", [(True, True, 2), (False, True, 1), (True, False, 0)])
def test_interactive_pt_frames(scene, checker, denoise, tone):
    import mrpnn_b200 as M
    W = 48
    ori, up, right = view_frame()
    viewer = M.Viewer(scene.vol, W, W, checkerboard=checker)
    for k in range(4):
        view = scene.vol.make_view((W, W), ori, up, right, LIGHT, scene.g, scene.alpha, multiScatter=64, seed=3)
        t0 = viewer.target.cpu().numpy()
        h0 = viewer.histo.cpu().numpy()
        fnum, flip = viewer.frame_num, viewer.flip
        img = viewer.frame(view, M.VolumeRender.PT, tone=tone, denoise=denoise, exposure=1.5)
        t1 = viewer.target.cpu().numpy()
        h1 = viewer.histo.cpu().numpy()
        ov = O.make_view(W, W, ori, up, right, LIGHT, alpha=scene.alpha, g=scene.g, multi_scatter=64, seed=3,
                         frame=k)
        ot, oh = O.frame_pt(scene.orc, ov, fnum // 2 if checker else fnum, int(checker), flip, t0, h0)
        same = np.isclose(t1, ot, rtol=1e-5, atol=1e-7).all(axis=-1)
        assert same.mean() > 0.9
        np.testing.assert_allclose(h1[same], oh[same], rtol=1e-5, atol=1e-6)
        ref, _ = O.frame_finish(t1, h1, fnum, flip, 0, int(denoise), 1.5, tone)
        d = np.abs(_channels(img) - _channels(ref))
        assert d.max() <= 1 and (d == 0).mean() > 0.99
        assert np.all((img >> 24) == 0xFF)


def test_interactive_mrpnn_checkerboard(scene):
    import mrpnn_b200 as M
    W = 40
    ori, up, right = view_frame()
    viewer = M.Viewer(scene.vol, W, W, checkerboard=True)
    view = scene.vol.make_view((W, W), ori, up, right, LIGHT, scene.g, scene.alpha, seed=1)
    viewer.target.fill_(-1.0)
    img = viewer.frame(view, M.VolumeRender.MRPNN, tone=2)
    t = viewer.target.cpu().numpy()
    rows, cols = np.indices((W, W))
    sel = (rows + cols + 0) % 2 == 0
    assert np.all(t[~sel] == -1.0)                    # unselected pixels keep their value
    assert np.all(t[sel] >= 0) and np.isfinite(t[sel]).all()
    ref, _ = O.frame_finish(t, viewer.histo.cpu().numpy(), 0, 0, 1, 0, 1.0, 2)
    d = np.abs(_channels(img) - _channels(ref))
    assert d.max() <= 1 and (d == 0).mean() > 0.99
