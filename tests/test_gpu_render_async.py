"""mrp_render_start / mrp_render_wait: started renders (results alternating
between two device buffers, copied out on a second stream) must give the
same images, bit for bit, as mrp_render of the same views -- in pinned host
and device outputs, across precisions, render types and a size change while
renders are in flight, and mixed with synchronous calls."""
import numpy as np
import pytest

from tests.gpu_scene import LIGHT, view_frame

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def vol():
    import mrpnn_b200 as M
    M.init()
    v = M.VolumeRender(64)
    v.generate_fbm(0, 4.0)
    v.Update()
    v.SetScatterRate(0.99)
    v.SetSky(0.05)
    v.SetBakeResolution(48)
    return v


def _views(v, sizes):
    ori, up, right = view_frame()
    return [v.make_view(s, ori, up, right, LIGHT, 0.857, 64.0, multiScatter=32, spp=2, seed=3, frame_offset=k)
            for k, s in enumerate(sizes)]


def _pinned(shape):
    import torch
    return torch.empty(shape, dtype=torch.float32).pin_memory().numpy()


def test_started_renders_match_sync(vol):
    import torch

    import mrpnn_b200 as M
    sizes = [(48, 48), (64, 40), (48, 48), (96, 96), (32, 32), (96, 96)]   # grows while renders are in flight
    for prec in (M.FP32, M.BF16, M.FP8):
        vol.SetPrecision(prec)
        views = _views(vol, sizes)
        ref = [vol.render_view(w, M.VolumeRender.MRPNN, 1, np.empty((w.height, w.width, 4), np.float32))
               for w in views]
        outs = []
        for k, w in enumerate(views):
            o = _pinned((w.height, w.width, 4)) if k % 2 == 0 else torch.empty((w.height, w.width, 4),
                                                                              dtype=torch.float32, device="cuda")
            outs.append(vol.render_view_start(w, M.VolumeRender.MRPNN, 1, o))
        vol.render_wait()
        for a, b in zip(outs, ref):
            a = a.cpu().numpy() if hasattr(a, "cpu") else a
            assert (b[..., 3] > 0).any()
            np.testing.assert_array_equal(_bits(a), _bits(b))
    vol.SetPrecision(M.FP32)


def test_started_tracer_and_mixed_sync(vol):
    import mrpnn_b200 as M
    views = _views(vol, [(32, 32)] * 4)
    ref = [vol.render_view(w, M.VolumeRender.PT, 2, np.empty((32, 32, 4), np.float32)) for w in views]
    outs = [_pinned((32, 32, 4)) for _ in views]
    vol.render_view_start(views[0], M.VolumeRender.PT, 2, outs[0])
    vol.render_view_start(views[1], M.VolumeRender.PT, 2, outs[1])
    # a synchronous render in between waits for the started ones first
    mid = vol.render_view(views[2], M.VolumeRender.PT, 2, np.empty((32, 32, 4), np.float32))
    vol.render_view_start(views[2], M.VolumeRender.PT, 2, outs[2])
    vol.render_view_start(views[3], M.VolumeRender.PT, 2, outs[3])
    vol.render_wait()
    np.testing.assert_array_equal(_bits(mid), _bits(ref[2]))
    for a, b in zip(outs, ref):
        np.testing.assert_array_equal(_bits(a), _bits(b))
    vol.render_wait()   # nothing in flight: returns at once


def test_frame_loop_with_keep_newest(vol):
    """start(k); wait(keep=1); frame k - 1 is complete in its buffer while
    frame k is still in flight (two pinned buffers alternate)."""
    import mrpnn_b200 as M
    vol.SetPrecision(M.BF16)
    views = _views(vol, [(64, 64)] * 6)
    ref = [vol.render_view(w, M.VolumeRender.MRPNN, 1, np.empty((64, 64, 4), np.float32)) for w in views]
    bufs = [_pinned((64, 64, 4)) for _ in range(2)]
    for k, w in enumerate(views):
        vol.render_view_start(w, M.VolumeRender.MRPNN, 1, bufs[k % 2])
        if k:
            vol.render_wait(keep=1)
            np.testing.assert_array_equal(_bits(bufs[(k - 1) % 2]), _bits(ref[k - 1]))
    vol.render_wait()
    np.testing.assert_array_equal(_bits(bufs[(len(views) - 1) % 2]), _bits(ref[-1]))
    vol.SetPrecision(M.FP32)
