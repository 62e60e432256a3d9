"""Parity at the benchmarked configurations, not only at the small test scenes.

* Predictor, FP32 drop-in: the headline frame -- 1024x1024 over the 512^3 fBm
  cloud (seed 1, base frequency 6, 6 octaves, gain 0.5), 9-level pyramid,
  extinction 64, albedo 0.99, g 0.857, light normalize(0.3, 0.8, 0.5), 45
  degree camera at (0.75, 0.75, 0.75).  The GPU renders the whole frame; the
  oracle (pinned to the reference's own NNPredict, core/render.cuh:808-875)
  evaluates 4,096 sampled pixels of it (2,048 of them among the hit pixels).
  Bar: the same pixels hit, and 99.9 % of the sampled pixels within 1e-4
  relative (+1e-6 absolute), the FP32 predictor's contract.  The same for the
  1920x1080 view of the precision form (2,048 sampled pixels).
* Tracer: the tracer workload -- 128^3 fBm (seed 0, base frequency 4),
  256x256, 16 spp, <= 256 bounces, NEE through the 768^3 baked transmittance
  grid, against the oracle's CalculateRadiance (core/render.cuh:535-597) over
  the whole frame with the same Philox streams and the GPU's baked grid.
  Bar: per-pixel z-score |z| < 4 for 99.9 % of the pixels, mean z within 0.1.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_scene import LIGHT, Scene, view_frame

pytestmark = pytest.mark.gpu

MLP_RTOL = 1e-4
MLP_ATOL = 1e-6


def test_headline_frame_fp32_matches_oracle():
    import mrpnn_b200 as M
    sc = Scene(R=512, seed=1, freq=6.0, alpha=64.0, g=0.857, sr=0.99, sky=0.05)
    W = 1024
    ori, up, right = view_frame()
    img = sc.vol.Render((W, W), ori, up, right, LIGHT, M.VolumeRender.MRPNN, sc.g, sc.alpha, sampleNum=1,
                        seed=3).reshape(-1, 4)
    hit = np.flatnonzero(img[:, 3] > 0)
    assert hit.size > 400_000                      # the cloud fills about half of the frame
    rng = np.random.default_rng(512)
    px = np.unique(np.concatenate([rng.choice(hit, 2048, replace=False),
                                   rng.choice(W * W, 2048, replace=False)])).astype(np.int32)
    view = O.make_view(W, W, ori, up, right, LIGHT, alpha=sc.alpha, g=sc.g, seed=3, frame=0)
    ref = O.predict_pixels(sc.orc, view, px)
    got = img[px]
    np.testing.assert_array_equal(got[:, 3] > 0, ref[:, 3] > 0)
    ok = np.isclose(got, ref, rtol=MLP_RTOL, atol=MLP_ATOL).all(axis=1)
    assert ok.mean() >= 0.999, (ok.mean(), px[~ok][:5])
    rel = np.abs(got[:, :3] - ref[:, :3]) / np.maximum(np.abs(ref[:, :3]), 1e-6)
    assert np.median(rel) < 1e-5

    # the precision form's second view: 1920x1080, the same 45 degree vertical
    # field of view (right scaled by 16/9), non-square rows and columns
    Wd, Hd = 1920, 1080
    right_w = (right * np.float32(16.0 / 9.0)).astype(np.float32)
    img = sc.vol.Render((Wd, Hd), ori, up, right_w, LIGHT, M.VolumeRender.MRPNN, sc.g, sc.alpha, sampleNum=1,
                        seed=4).reshape(-1, 4)
    hit = np.flatnonzero(img[:, 3] > 0)
    px = np.unique(np.concatenate([rng.choice(hit, 1024, replace=False),
                                   rng.choice(Wd * Hd, 1024, replace=False)])).astype(np.int32)
    view = O.make_view(Wd, Hd, ori, up, right_w, LIGHT, alpha=sc.alpha, g=sc.g, seed=4, frame=0)
    ref = O.predict_pixels(sc.orc, view, px)
    got = img[px]
    np.testing.assert_array_equal(got[:, 3] > 0, ref[:, 3] > 0)
    ok = np.isclose(got, ref, rtol=MLP_RTOL, atol=MLP_ATOL).all(axis=1)
    assert ok.mean() >= 0.999, (ok.mean(), px[~ok][:5])


# the tensor-core forms against the FP32 drop-in on the same frame
# (tests/test_gpu_tensor_core.py states the same bounds against FP64)
TC_REL_RMS = {"BF16": 0.02, "FP8": 0.08}


@pytest.mark.parametrize("prec", ["BF16", "FP8"])
def test_headline_frame_tensor_core_forms(prec):
    """The precision forms on the headline frame (1024x1024 over the 512^3
    cloud): the same pixels hit at the same distances as the FP32 form (the
    march is shared and exact), and the radiance of the hit pixels within the
    form's relative RMS of the FP32 form's, with the fp16 features of the
    texture-unit gather (the default) and of the software gather."""
    import mrpnn_b200 as M
    sc = Scene(R=512, seed=1, freq=6.0, alpha=64.0, g=0.857, sr=0.99, sky=0.05)
    W = 1024
    ori, up, right = view_frame()

    def frame():
        return sc.vol.Render((W, W), ori, up, right, LIGHT, M.VolumeRender.MRPNN, sc.g, sc.alpha, sampleNum=1,
                             seed=3).reshape(-1, 4)
    ref = frame()
    hit = ref[:, 3] > 0
    sc.vol.SetPrecision(getattr(M, prec))
    try:
        for hw in (True, False):
            sc.vol.SetGatherFilter(hw)
            got = frame()
            np.testing.assert_array_equal(got[:, 3], ref[:, 3])
            rms = np.sqrt(np.mean((got[hit, :3] - ref[hit, :3]) ** 2)) / np.sqrt(np.mean(ref[hit, :3] ** 2))
            print(f"{prec} gather_filter={int(hw)}: rel RMS vs FP32 {rms:.4f} over {hit.sum()} hit pixels")
            assert rms < TC_REL_RMS[prec]
            np.testing.assert_array_equal(got[~hit], ref[~hit])   # sky pixels: the same constant
    finally:
        sc.vol.SetPrecision(M.FP32)
        sc.vol.SetGatherFilter(True)


@pytest.mark.parametrize("hw_filter", [False, True], ids=["software", "texture"])
def test_tracer_workload_zscore(hw_filter):
    """The C1 tracer workload against the oracle's tracer, per pixel.  With
    the texture unit's filters (tracer_filter) the GPU's density and NEE
    values differ from the oracle's by the unit's 8-bit weights, so its
    paths part from the oracle's and the comparison is between two
    independent estimates: the same bars hold."""
    import mrpnn_b200 as M
    sc = Scene(R=128, seed=0, freq=4.0, alpha=64.0, g=0.857, sr=0.99, sky=0.05, bake_res=768)
    W, spp, bounces = 256, 16, 256
    ori, up, right = view_frame()
    sc.vol.SetTracerFilter(hw_filter)
    try:
        got = sc.vol.Render((W, W), ori, up, right, LIGHT, M.VolumeRender.PT, sc.g, sc.alpha, multiScatter=bounces,
                            sampleNum=1, spp=spp, seed=9).reshape(-1, 4)
    finally:
        sc.vol.SetTracerFilter(False)
    view = O.make_view(W, W, ori, up, right, LIGHT, alpha=sc.alpha, g=sc.g, multi_scatter=bounces, spp=spp,
                       seed=9, frame=0)
    rgba, s, s2 = O.trace_pixels(sc.orc, view, np.arange(W * W, dtype=np.int32))
    mean = s / spp
    var = np.maximum(s2 / spp - mean ** 2, 0) * spp / (spp - 1)
    se = np.sqrt(2 * var / spp) + 1e-7
    z = (got[:, :3] - mean) / se
    zf = z[np.isfinite(z)]
    assert np.mean(np.abs(zf) < 4) >= 0.999, np.mean(np.abs(zf) < 4)
    assert abs(zf.mean()) < 0.1, zf.mean()
    # the frame is not trivially sky: most pixels see the cloud
    assert np.mean(rgba[:, 3] > 0) > 0.3
    assert got[:, 3].min() >= 0 and got[:, 3].max() <= 1
