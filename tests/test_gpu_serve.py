"""The serving loop (mrp_serve_*) on the GPU: every result of a mixed,
queued, batched request stream equals mrp_render of the same view alone.

The server runs the same kernels as mrp_render (TR mips per request, first
hit, gather) and evaluates the network of several requests in one launch;
each row of the network is computed independently of the batch, so the
results must agree to the last bit (checked with a 1e-6 relative bound)."""
import numpy as np
import pytest

from tests.gpu_scene import LIGHT, view_frame

pytestmark = pytest.mark.gpu

SAME_RTOL = 1e-6
SAME_ATOL = 1e-7


def _volumes(M, precision):
    vols = []
    for R, seed, freq, alpha in ((64, 10, 4.0, 32.0), (96, 11, 5.0, 96.0), (128, 12, 6.0, 200.0)):
        v = M.VolumeRender(R)
        v.generate_fbm(seed, freq)
        v.Update()
        v.SetScatterRate(0.99)
        v.SetSky(0.05)
        v.SetPrecision(precision)
        vols.append((v, alpha))
    return vols


def _requests(M, vols, n, rng):
    reqs = []
    for i in range(n):
        v, alpha = vols[i % len(vols)]
        W, H = [(64, 64), (96, 64), (128, 128), (80, 112)][rng.integers(4)]
        r = rng.uniform(0.8, 2.0)
        th, ph = rng.uniform(0, 2 * np.pi), rng.uniform(0.2, 1.3)
        pos = (r * np.sin(ph) * np.cos(th), r * np.cos(ph), r * np.sin(ph) * np.sin(th))
        ori, up, right = view_frame(45.0, pos)
        L = rng.normal(size=3)
        L = (L / np.linalg.norm(L)).astype(np.float32)
        view = v.make_view((W, H), ori, up, right, L, g=0.857, alpha=alpha, seed=int(rng.integers(1 << 30)),
                           frame_offset=int(rng.integers(4)))
        reqs.append((v, view))
    return reqs


@pytest.mark.parametrize("precision", ["BF16", "FP8", "FP32"])
def test_serve_mix_equals_alone(precision):
    import mrpnn_b200 as M
    M.init()
    prec = getattr(M, precision)
    vols = _volumes(M, prec)
    rng = np.random.default_rng(7)
    reqs = _requests(M, vols, 14, rng)
    alone = [v.render_view(view, M.VolumeRender.MRPNN, 1, np.empty((view.height, view.width, 4), np.float32))
             for v, view in reqs]
    srv = M.Server(max_slots=4, precision=prec, slot_pixels=128 * 128 if precision == "BF16" else 0)
    try:
        tickets = [srv.submit(v, view) for v, view in reqs]
        times = []
        for k, t in enumerate(tickets):
            out, tm = srv.wait(t)
            np.testing.assert_allclose(out, alone[k], rtol=SAME_RTOL, atol=SAME_ATOL)
            assert tm["submit_ms"] <= tm["admit_ms"] <= tm["features_ms"] <= tm["network_ms"] <= tm["done_ms"]
            times.append(tm)
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        # continuous batching, not a queue: requests were on the device at the
        # same time (their intervals from admission to result overlap) ...
        overlaps = sum(1 for i in range(len(times)) for j in range(i + 1, len(times))
                       if times[i]["admit_ms"] < times[j]["done_ms"] and
                       times[j]["admit_ms"] < times[i]["done_ms"])
        assert overlaps >= 3, overlaps
        if prec != M.FP32:
            # ... and network launches carried several requests each
            assert st["batched_requests"] == len(reqs)
            assert st["max_batch"] >= 2 and st["batches"] < len(reqs), st
    finally:
        srv.close()


def test_serve_device_output_and_budget():
    import torch
    import mrpnn_b200 as M
    M.init()
    vols = _volumes(M, M.BF16)
    rng = np.random.default_rng(8)
    (v, view), = _requests(M, vols[:1], 1, rng)
    alone = v.render_view(view, M.VolumeRender.MRPNN, 1, np.empty((view.height, view.width, 4), np.float32))
    srv = M.Server(max_slots=2, precision=M.BF16, memory_budget=128 << 20)
    try:
        out = torch.empty((view.height, view.width, 4), dtype=torch.float32, device="cuda")
        got, _ = srv.wait(srv.submit(v, view, out))
        np.testing.assert_allclose(got.cpu().numpy(), alone, rtol=SAME_RTOL, atol=SAME_ATOL)
        big = v.make_view((2048, 2048), *view_frame(), LIGHT, alpha=32.0)
        with pytest.raises(M.MrpError) as e:
            srv.submit(v, big)
        assert e.value.status == M.api.ERR_BUDGET
        assert srv.stats()["peak_bytes"] <= 128 << 20
    finally:
        srv.close()
