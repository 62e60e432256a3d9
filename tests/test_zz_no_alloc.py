"""mrp_predict_features_noalloc (no counterpart in the reference) against
mrp_predict_features on the same host inputs, both through the C ABI.

The no-allocation entry point is for callers that must not allocate device
memory while they render (a frame loop that cannot take the device-wide
synchronisation of cudaFree, or a process whose memory pool already holds
the HBM).  It runs the same network kernels as mrp_predict_features, with
its staging, output, tile counter and error flag in the library's fixed
device array.  So two calls in a row must each match the allocating call
within the predictor's test tolerance, and the library's count of
allocation calls (and the device memory in use) must not change across
calls.  The file is named to be collected last."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MLP_RTOL = 1e-4      # same bound as the FP32 predictor parity tests
MLP_ATOL = 1e-6


def _features(n, seed):
    rng = np.random.default_rng(seed)
    feat = np.concatenate([rng.uniform(0, 1.5, (n, 192)), rng.uniform(0, 1, (n, 192)),
                           rng.uniform(0, 3, (n, 192))], 1).astype(np.float32)
    gam = rng.uniform(0, np.pi, n).astype(np.float32)
    return feat, gam


@pytest.mark.parametrize("precision", ["FP32", "BF16", "FP8"])
def test_noalloc_matches_predict_features(precision):
    import mrpnn_b200 as M
    M.init()
    prec = getattr(M, precision)
    feat, gam = _features(1500, 31)
    sr = (0.99, 0.9, 0.8)
    ref = M.predict_features(feat, gam, 0.857, sr, precision=prec)
    for _ in range(2):
        got = M.predict_features_noalloc(feat, gam, 0.857, sr, precision=prec)
        np.testing.assert_allclose(got, ref, rtol=MLP_RTOL, atol=MLP_ATOL)


def test_noalloc_full_capacity_and_rejects_more():
    import mrpnn_b200 as M
    M.init()
    n = M.NOALLOC_MAX_POINTS
    feat, gam = _features(n, 32)
    ref = M.predict_features(feat, gam, 0.5, (1, 1, 1), precision=M.BF16)
    got = M.predict_features_noalloc(feat, gam, 0.5, (1, 1, 1), precision=M.BF16)
    np.testing.assert_allclose(got, ref, rtol=MLP_RTOL, atol=MLP_ATOL)
    feat, gam = _features(n + 1, 33)
    with pytest.raises(M.MrpError, match="split the batch"):
        M.predict_features_noalloc(feat, gam, 0.5, (1, 1, 1))


def test_noalloc_makes_no_allocation_call():
    """The library counts every cudaMalloc / cudaMallocAsync / cudaMallocHost
    and free it makes; the no-allocation entry point must add none, not even
    one freed again before it returns.  Device-wide free memory is checked as
    well, as a second witness."""
    import torch
    import mrpnn_b200 as M
    M.init()
    feat, gam = _features(1024, 34)
    M.predict_features_noalloc(feat, gam, 0.857, (1, 1, 1), precision=M.BF16)   # first call: address lookup
    torch.cuda.synchronize()
    calls = M.debug_alloc_calls()
    before = torch.cuda.mem_get_info()[0]
    for prec in (M.FP32, M.BF16, M.FP8, M.BF16):
        M.predict_features_noalloc(feat, gam, 0.857, (1, 1, 1), precision=prec)
    assert M.debug_alloc_calls() == calls
    assert torch.cuda.mem_get_info()[0] == before
    v = M.VolumeRender(16)                      # a volume handle allocates: the counter sees it
    assert M.debug_alloc_calls() > calls
    del v
