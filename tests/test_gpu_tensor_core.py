"""Tensor-core (tcgen05) forms of the MRPNN MLP.

1. The operand layout / descriptors: one tcgen05.mma chain against numpy on
   operands rounded exactly like the kernel rounds them.
2. BF16 and FP8-E4M3 networks against the FP64 evaluation of the same
   network on the same features (the error the precision costs), and against
   the FP32 drop-in.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# Error bounds of the reduced-precision forms against the FP64 network:
# relative RMS over all outputs, and the largest absolute error in units of
# the RMS output (single outputs near 0 make plain max-relative meaningless).
BF16_REL_RMS, BF16_NORM_MAX = 0.02, 0.15
FP8_REL_RMS, FP8_NORM_MAX = 0.08, 0.60


def _round(x, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(dtype).float().numpy()


@pytest.mark.parametrize("n,k", [(16, 16), (32, 64), (64, 128), (128, 128), (16, 32), (128, 32)])
def test_tc_gemm_bf16(n, k):
    import torch
    import mrpnn_b200 as M
    rng = np.random.default_rng(n * 1000 + k)
    A = rng.normal(size=(128, k)).astype(np.float32)
    B = rng.normal(size=(n, k)).astype(np.float32)
    D = M.api.tc_gemm_check(A, B, fp8=False)
    ref = _round(A, torch.bfloat16).astype(np.float64) @ _round(B, torch.bfloat16).astype(np.float64).T
    np.testing.assert_allclose(D, ref, rtol=1e-4, atol=1e-4 * np.sqrt(k))


@pytest.mark.parametrize("n,k", [(16, 32), (64, 64), (128, 128)])
def test_tc_gemm_fp8(n, k):
    import torch
    import mrpnn_b200 as M
    rng = np.random.default_rng(n * 7 + k)
    A = rng.uniform(-4, 4, size=(128, k)).astype(np.float32)
    B = rng.uniform(-4, 4, size=(n, k)).astype(np.float32)
    D = M.api.tc_gemm_check(A, B, fp8=True)
    ref = _round(A, torch.float8_e4m3fn).astype(np.float64) @ _round(B, torch.float8_e4m3fn).astype(np.float64).T
    np.testing.assert_allclose(D, ref, rtol=1e-4, atol=1e-3 * np.sqrt(k))


def _features(n, seed):
    """Features gathered from a real scene (the distribution the network sees)."""
    from tests.gpu_scene import LIGHT, Scene, view_frame
    sc = Scene(R=64, seed=seed)
    W = int(np.ceil(np.sqrt(n * 2.2)))
    ori, up, right = view_frame()
    view = sc.vol.make_view((W, W), ori, up, right, LIGHT, sc.g, sc.alpha, seed=seed)
    _, aux, feat = sc.vol.predict_debug(view)
    hit = aux[:, 3] > 0
    return feat[hit][:n], aux[hit, 4][:n]


@pytest.fixture(scope="module")
def feats():
    return _features(3000, 4)


def _rel_errors(got, ref):
    scale = np.sqrt(np.mean(ref ** 2))
    rms = np.sqrt(np.mean((got - ref) ** 2)) / scale
    return rms, np.abs(got - ref).max() / scale


@pytest.mark.parametrize("sr", [(0.99 / 1.001,) * 3, (0.99, 0.9, 0.8)])
def test_mlp_bf16_vs_fp64(feats, sr):
    import mrpnn_b200 as M
    feat, gam = feats
    got = M.predict_features(feat, gam, 0.857, sr, precision=M.BF16)
    ref = O.mlp_f64(feat, gam, 0.857, sr)
    rms, mx = _rel_errors(got, ref)
    print(f"BF16: rel RMS {rms:.4f}, max |err| / RMS {mx:.4f}")
    assert rms < BF16_REL_RMS and mx < BF16_NORM_MAX


@pytest.mark.parametrize("sr", [(0.99 / 1.001,) * 3, (0.99, 0.9, 0.8)])
def test_mlp_fp8_vs_fp64(feats, sr):
    import mrpnn_b200 as M
    feat, gam = feats
    got = M.predict_features(feat, gam, 0.857, sr, precision=M.FP8)
    ref = O.mlp_f64(feat, gam, 0.857, sr)
    rms, mx = _rel_errors(got, ref)
    print(f"FP8: rel RMS {rms:.4f}, max |err| / RMS {mx:.4f}")
    assert rms < FP8_REL_RMS and mx < FP8_NORM_MAX


def test_mlp_tc_partial_tiles():
    """n not a multiple of the 128-row tile, and n smaller than one tile."""
    import mrpnn_b200 as M
    rng = np.random.default_rng(3)
    for n in (1, 77, 129, 300):
        feat = rng.uniform(0, 1.5, (n, 576)).astype(np.float32)
        gam = rng.uniform(0, 3, n).astype(np.float32)
        got = M.predict_features(feat, gam, 0.5, (1, 1, 1), precision=M.BF16)
        ref = O.mlp_f64(feat, gam, 0.5, (1, 1, 1))
        rms, _ = _rel_errors(got, ref)
        assert rms < BF16_REL_RMS, (n, rms)


@pytest.mark.parametrize("prec", ["bf16", "fp8"])
def test_render_tc_close_to_fp32(prec):
    import mrpnn_b200 as M
    from tests.gpu_scene import LIGHT, Scene, view_frame
    sc = Scene(R=64)
    ori, up, right = view_frame()
    W = 64
    sc.vol.SetPrecision(M.FP32)
    a = sc.vol.Render((W, W), ori, up, right, LIGHT, M.VolumeRender.MRPNN, sc.g, sc.alpha, sampleNum=1, seed=2)
    sc.vol.SetPrecision(M.BF16 if prec == "bf16" else M.FP8)
    b = sc.vol.Render((W, W), ori, up, right, LIGHT, M.VolumeRender.MRPNN, sc.g, sc.alpha, sampleNum=1, seed=2)
    np.testing.assert_array_equal(a[..., 3], b[..., 3])     # same hits / distances
    hit = a[..., 3] > 0
    rms = np.sqrt(np.mean((a[hit, :3] - b[hit, :3]) ** 2)) / np.sqrt(np.mean(a[hit, :3] ** 2))
    print(f"{prec} render rel RMS vs FP32: {rms:.4f}")
    assert rms < (BF16_REL_RMS if prec == "bf16" else FP8_REL_RMS)
