"""mrp_render_views: several views of one volume, one batched network
launch; each image must equal mrp_render of that view alone (same kernels,
same per-pixel streams; 1e-6 relative bound)."""
import numpy as np
import pytest

from tests.gpu_scene import LIGHT, view_frame

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["BF16", "FP8", "FP32"])
def test_views_equal_single_renders(precision):
    import mrpnn_b200 as M
    M.init()
    v = M.VolumeRender(96)
    v.generate_fbm(21, 5.0)
    v.Update()
    v.SetScatterRate(0.99)
    v.SetSky(0.05)
    v.SetPrecision(getattr(M, precision))
    rng = np.random.default_rng(4)
    views = []
    for k in range(7):
        d = rng.normal(size=3)
        pos = tuple(float(x) for x in rng.uniform(0.9, 1.8) * d / np.linalg.norm(d))
        ori, up, right = view_frame(45.0, pos)
        W, H = [(64, 64), (80, 48), (40, 72)][k % 3]
        views.append(v.make_view((W, H), ori, up, right, LIGHT, g=0.857, alpha=80.0, seed=k, frame_offset=k % 2))
    got = v.render_views(views)
    for view, img in zip(views, got):
        alone = v.render_view(view, M.VolumeRender.MRPNN, 1, np.empty((view.height, view.width, 4), np.float32))
        np.testing.assert_allclose(img, alone, rtol=1e-6, atol=1e-7)
    hit = v.render_views(views[:1])[0]
    np.testing.assert_allclose(hit, got[0], rtol=1e-6, atol=1e-7)


def test_views_must_share_light():
    import mrpnn_b200 as M
    M.init()
    v = M.VolumeRender(32)
    v.generate_fbm(1, 4.0)
    v.Update()
    ori, up, right = view_frame()
    a = v.make_view((16, 16), ori, up, right, LIGHT, alpha=16.0)
    b = v.make_view((16, 16), ori, up, right, -LIGHT, alpha=16.0)
    with pytest.raises(M.MrpError, match="share the light"):
        v.render_views([a, b])
