"""Benchmark of the MRPNN render path on B200.

Workload (the headline configuration): MRPNN predictor frames of 1024x1024 over
a 512^3 fp32 fBm cloud (seed 1, base frequency 6, 6 octaves, gain 0.5),
9-level pyramid, extinction 64, albedo 0.99, g 0.857, light
normalize(0.3, 0.8, 0.5), sky 0.05, 45 degree camera at (0.75, 0.75, 0.75),
one predictor evaluation per pixel.  A step is one frame.

  python bench.py [--gpus N --steps K --warmup W] [--precision fp32|bf16|fp8]
  python bench.py --impl reference        # CPU port of the reference path

N > 1 runs one process per GPU (torchrun); each GPU renders its own frames
from its own replica of the volume (the path shards by frame, no collective):
value = frames of all ranks / max over ranks of the device time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1024^2 MRPNN frames/s"
UNIT = "frames/s"
W = H = 1024
RES = 512
SCENE = dict(seed=1, freq=6.0, octaves=6, gain=0.5, alpha=64.0, g=0.857, albedo=0.99, sky=0.05,
             light=(0.3, 0.8, 0.5), cam=(0.75, 0.75, 0.75), fov=45.0)
GATHER_BYTES_PER_PIXEL = 192 * (8 + 8 + 2 * 4) * 4     # density + TR trilinear, 2 LUT bilinear, fp32


def light():
    L = np.asarray(SCENE["light"], np.float32)
    return (L / np.float32(np.sqrt(np.float32(np.dot(L, L))))).astype(np.float32)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], p["bf16_tflops"], "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n):
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        # one process per GPU over NCCL; gloo only where no GPU is visible
        # (the CPU tests of this rank logic)
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_scene_from_gpu(vol):
    """Host copies of the GPU resources (bit-identical to the oracle's own
    construction, which tests/test_gpu_resources.py checks)."""
    import mrpnn_b200 as M
    from oracle import oracle as O
    mips = np.concatenate([vol.read(M.api.RES_MIP, m) for m in range(9)])
    tr = np.concatenate([vol.read(M.api.RES_TR, i) for i in range(8)])
    return O.SceneBuf(vol.read(M.api.RES_DENSITY), RES, vol.max_density, mips, tr, vol.read(M.api.RES_LUT),
                      scatter_rate=(SCENE["albedo"],) * 3, sky=(SCENE["sky"],) * 3)


def cpu_scene_oracle():
    """The scene built by the CPU port alone (reference arm: no GPU code)."""
    from oracle import oracle as O
    vol = O.fbm_volume(RES, SCENE["seed"], SCENE["freq"], SCENE["octaves"], SCENE["gain"])
    md = O.lib().orc_max_density(vol, vol.size)
    mips = O.build_pyramid(vol, RES)
    tr = O.tr_mips(mips, SCENE["alpha"], light())
    _, tex = O.lut_rows_needed()
    lut = np.zeros(512 * 512, np.float32)
    lut[tex] = O.hg_lut_texels(SCENE["g"], 0, tex)
    return O.SceneBuf(vol, RES, md, mips, tr, lut, scatter_rate=(SCENE["albedo"],) * 3, sky=(SCENE["sky"],) * 3)


def view_vectors():
    import mrpnn_b200 as M
    ori, up, right = M.camera_frame(SCENE["cam"])
    s = np.float32(np.tan(np.deg2rad(SCENE["fov"]) / 2))
    return ori, (up * s).astype(np.float32), (right * s).astype(np.float32)


def time_cpu_predict(sc, n_pix, seed=0, reps=1, want=False):
    """Oracle predictor on a random sample of the 1024^2 frame -> pixels/s
    (and, with want, the sampled pixel indices and their RGBA)."""
    from oracle import oracle as O
    ori, up, right = view_vectors()
    view = O.make_view(W, H, ori, up, right, light(), alpha=SCENE["alpha"], g=SCENE["g"], seed=seed, frame=0)
    rng = np.random.default_rng(seed)
    px = rng.choice(W * H, n_pix, replace=False).astype(np.int32)
    t0 = time.perf_counter()
    for _ in range(reps):
        rgba = O.predict_pixels(sc, view, px)
    dt = time.perf_counter() - t0
    if want:
        return n_pix * reps / dt, dt, px, rgba
    return n_pix * reps / dt, dt


def time_torch_network(sc, hits_per_frame, n_pix=16384, min_s=3.0):
    """The network alone as a batched PyTorch CPU model (oracle/torch_mlp.py)
    on the stencil features of n_pix sampled hit pixels of the frame ->
    network pixels/s and the frames/s that rate gives at the frame's hit
    count; torch's own thread count."""
    import torch

    from oracle import oracle as O
    from oracle.torch_mlp import RadiancePredictor
    ori, up, right = view_vectors()
    view = O.make_view(W, H, ori, up, right, light(), alpha=SCENE["alpha"], g=SCENE["g"], seed=0, frame=0)
    px = np.random.default_rng(5).choice(W * H, 4 * n_pix, replace=False).astype(np.int32)
    rgba, feat, gam, hit = O.predict_pixels(sc, view, px, want_features=True)
    sel = np.flatnonzero(hit[:, 3] > 0)[:n_pix]
    feat, gam = feat[sel], gam[sel]
    model = RadiancePredictor()
    sr = (SCENE["albedo"] / 1.001,) * 3
    model(feat[:256], gam[:256], SCENE["g"], sr)   # warm-up
    t0, reps = time.perf_counter(), 0
    while True:
        model(feat, gam, SCENE["g"], sr)
        reps += 1
        dt = time.perf_counter() - t0
        if dt >= min_s:
            break
    pps = reps * len(sel) / dt
    return {"value": pps, "unit": "network pixels/s", "cores": torch.get_num_threads(), "kind": "port",
            "frames_per_s_network_only": pps / max(1, hits_per_frame),
            "sample": f"{reps} passes over the features of {len(sel)} hit pixels ({dt:.1f} s), batched PyTorch "
                      f"float32 CPU port of RadiancePredictInternal"}


def frame_parity(vol, px, ref, local):
    """The GPU's FP32 frame of the CPU baseline's view (seed 0, frame 0)
    against the oracle's pixels px (RGBA ref): the FP32 predictor's 1e-4
    relative contract, checked at the benchmarked size."""
    import torch

    import mrpnn_b200 as M
    ori, up, right = view_vectors()
    prec = vol.GetPrecision()
    vol.SetPrecision(M.FP32)
    try:
        view = vol.make_view((W, H), ori, up, right, light(), SCENE["g"], SCENE["alpha"], seed=0, frame_offset=0)
        out = torch.empty((H, W, 4), dtype=torch.float32, device=f"cuda:{local}")
        vol.render_view(view, M.VolumeRender.MRPNN, 1, out)
        got = out.reshape(-1, 4).cpu().numpy()[px]
    finally:
        vol.SetPrecision(prec)
    ok = np.isclose(got, ref, rtol=1e-4, atol=1e-6).all(axis=1)
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-6)
    hit_g, hit_r = got[:, 3] > 0, ref[:, 3] > 0
    return {"form": "fp32", "pixels": int(px.size), "hit_pixels": int(hit_r.sum()),
            "hit_mismatch": int((hit_g != hit_r).sum()), "frac_within_1e-4_rel": float(ok.mean()),
            "max_rel": float(rel[:, :3].max()),
            "median_rel_hit": float(np.median(rel[hit_r, :3])) if hit_r.any() else 0.0,
            "tolerance": "rtol 1e-4 + atol 1e-6 per RGBA component (the FP32 predictor contract)",
            "oracle": "OpenMP CPU oracle, pinned bit for bit to the reference's own NNPredict compiled on the CPU"}


def omp_threads():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def run_reference(args, rank, world):
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    t0 = time.perf_counter()
    sc = cpu_scene_oracle()
    setup_s = time.perf_counter() - t0
    n_pix = args.ref_pixels
    for _ in range(args.warmup):
        time_cpu_predict(sc, max(256, n_pix // 8))
    secs = []
    for k in range(args.steps):
        _, dt = time_cpu_predict(sc, n_pix, seed=k + 1)
        secs.append(dt)
    pix_s = n_pix * len(secs) / float(np.sum(secs))
    fps = pix_s / (W * H)
    cores = omp_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": fps, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.mean(secs)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"MRPNN predictor, {W}x{H} frame, {RES}^3 fBm (seed 1, freq 6), FP32 MLP",
                   "sample": f"{n_pix} random pixels per step",
                   "step": "one step = the sampled pixels of one frame; ms_per_step is the measured time of that "
                           "sample; value = sampled pixels/s over all steps / pixels per frame",
                   "ms_per_full_frame": 1000.0 / fps},
        "cpu_baseline": {"value": fps, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{n_pix} random pixels of the {W}x{H} frame per step, scene setup {setup_s:.1f}s"},
        "e2e": {"value": fps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


TRACER = dict(res=128, seed=0, freq=4.0, size=256, spp=16, bounces=256, bake_res=768)


def run_tracer(args, local):
    """The delta-tracking path tracer on its own workload: 128^3 fBm (seed 0,
    freq 4), 256x256, 16 spp, <= 256 bounces, NEE through the 768^3 baked
    transmittance grid.  Returns a dict for the JSON line."""
    import torch

    import mrpnn_b200 as M
    vol = M.VolumeRender(TRACER["res"])
    vol.generate_fbm(TRACER["seed"], TRACER["freq"])
    vol.Update()
    vol.SetScatterRate(SCENE["albedo"])
    vol.SetSky(SCENE["sky"])
    vol.SetBakeResolution(TRACER["bake_res"])
    L = light()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    vol.Update_CachedTR(L, SCENE["alpha"])
    bake_s = time.perf_counter() - t0
    ori, up, right = view_vectors()
    n = TRACER["size"]
    view = vol.make_view((n, n), ori, up, right, L, SCENE["g"], SCENE["alpha"], multiScatter=TRACER["bounces"],
                         spp=TRACER["spp"], seed=7)
    out = torch.empty((n, n, 4), dtype=torch.float32, device=f"cuda:{local}")
    vol.render_view(view, M.VolumeRender.PT, 1, out)
    ms, trace_ms = [], []
    for k in range(args.tracer_steps):
        view.frame_offset = 10 + k
        vol.render_view(view, M.VolumeRender.PT, 1, out)
        ms.append(vol.last_render_ms())
        trace_ms.append(vol.last_render_stages()[0])   # the trace kernel of this timed frame
    trace_ms = float(np.mean(trace_ms))
    # work counters of the first timed frame (same streams; a separate,
    # instrumented launch that is not timed)
    view.frame_offset = 10
    cnt = vol.render_counters(view, M.VolumeRender.PT)   # bounces, fetches, NEE lookups, samples
    t = float(np.mean(ms))
    hbm, _, peak_kind = peaks()
    alg = (cnt[1] + cnt[2]) * 32 + n * n * 16
    ach = alg / (trace_ms / 1000.0) / 1e9
    res = {"workload": f"PT {n}x{n}, {TRACER['spp']} spp, <= {TRACER['bounces']} bounces, "
                       f"{TRACER['res']}^3 fBm (seed 0, freq 4), NEE via {TRACER['bake_res']}^3 baked TR",
           "ms_per_frame": t, "trace_kernel_ms": trace_ms, "samples_per_s": n * n * TRACER["spp"] / (t / 1000.0),
           "density_lookups_per_s": (cnt[1] + cnt[2]) / (trace_ms / 1000.0),
           "counters": {"bounces": cnt[0], "free_flight_fetches": cnt[1], "nee_lookups": cnt[2], "samples": cnt[3]},
           "bake_s": bake_s,
           "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                        "note": f"trace kernel of the timed frames; algorithmic bytes = (fetches + NEE lookups) x 32 B "
                                f"(8 fp32 texels) + 16 B/pixel; peak {peak_kind}; the 8 MiB volume is L2-resident"}}
    # the same frames with the texture unit's trilinear filter in the free
    # flight (tracer_filter 1, the reference's own tex3D filtering)
    vol.SetTracerFilter(True)
    view.frame_offset = 9
    vol.render_view(view, M.VolumeRender.PT, 1, out)   # builds the density texture
    ms_hw, tr_hw = [], []
    for k in range(args.tracer_steps):
        view.frame_offset = 10 + k
        vol.render_view(view, M.VolumeRender.PT, 1, out)
        ms_hw.append(vol.last_render_ms())
        tr_hw.append(vol.last_render_stages()[0])
    vol.SetTracerFilter(False)
    t_hw = float(np.mean(tr_hw))
    ach_hw = alg / (t_hw / 1000.0) / 1e9
    # the level the lookups are served from: the 8 MiB volume stays in L2
    # (and mostly L1); its ceiling is the measured rate of L2 reads
    l2 = M.api.measure_l2_rate()
    res["roofline"]["l2"] = {"peak": l2, "unit": "GB/s", "frac": ach / l2, "frac_hw_filter": ach_hw / l2,
                             "note": "same algorithmic bytes against the measured L2 read rate "
                                     "(mrp_measure_l2_rate, 64 MiB L2-resident buffer, L1 bypassed)"}
    res["hw_filter"] = {"ms_per_frame": float(np.mean(ms_hw)), "trace_kernel_ms": t_hw,
                        "samples_per_s": n * n * TRACER["spp"] / (float(np.mean(ms_hw)) / 1000.0),
                        "roofline": {"bound": "hbm", "achieved": ach_hw, "peak": hbm, "unit": "GB/s",
                                     "frac": ach_hw / hbm,
                                     "note": "same algorithmic bytes (the software path's counters); free-flight "
                                             "fetches through the texture unit"}}
    if args.tracer_cpu_frames > 0:
        res["cpu_baseline"] = time_cpu_tracer(vol, args.tracer_cpu_frames)
    return res


def time_cpu_tracer(vol, frames):
    """The oracle's CalculateRadiance (OpenMP) on the tracer workload: the
    same scene (the GPU's grid and baked NEE grid), the same spp and bounce
    limit, whole frames -> samples/s."""
    import mrpnn_b200 as M
    from oracle import oracle as O
    R = TRACER["res"]
    sc = O.SceneBuf(vol.read(M.api.RES_DENSITY), R, vol.max_density, baked=vol.read(M.api.RES_BAKED_TR),
                    baked_res=TRACER["bake_res"], scatter_rate=(SCENE["albedo"],) * 3, sky=(SCENE["sky"],) * 3)
    n = TRACER["size"]
    ori, up, right = view_vectors()
    px = np.arange(n * n, dtype=np.int32)
    t0 = time.perf_counter()
    for f in range(frames):
        ov = O.make_view(n, n, ori, up, right, light(), alpha=SCENE["alpha"], g=SCENE["g"],
                         multi_scatter=TRACER["bounces"], spp=TRACER["spp"], seed=7, frame=10 + f)
        O.trace_pixels(sc, ov, px)
    dt = time.perf_counter() - t0
    sps = frames * n * n * TRACER["spp"] / dt
    return {"value": sps, "unit": "samples/s", "cores": omp_threads(), "kind": "port",
            "ms_per_frame": dt / frames * 1000.0,
            "sample": f"{frames} whole {n}x{n} frames x {TRACER['spp']} spp ({dt:.1f} s), OpenMP oracle "
                      "CalculateRadiance with the baked NEE grid"}


SERVE = dict(volumes=16, sizes=(128, 256, 512), seeds=range(10, 26), alpha=(16.0, 256.0), freq=4.0, rate=200.0,
             images=((256, 256), (512, 512), (1024, 1024), (1920, 1080)), radius=(0.8, 2.0), budget=120 << 30,
             slots=16)


def run_serving(args, local):
    """Serving workload: 16 resident fBm volumes (edges drawn from 128/256/512,
    seeds 10-25, extinction 16-256), a seeded Poisson stream of MRPNN requests
    at 200 req/s with images drawn from 256^2 / 512^2 / 1024^2 / 1920x1080,
    random orbit cameras (radius 0.8-2) and random lights, BF16 network,
    120 GB admission budget.  Latency = submit -> result in the caller's
    (device) buffer, from the server's own clock."""
    import threading

    import torch

    import mrpnn_b200 as M
    rng = np.random.default_rng(2024)
    vols = []
    for seed in SERVE["seeds"]:
        R = int(rng.choice(SERVE["sizes"]))
        v = M.VolumeRender(R, storage="fp16")   # fp16 density grids
        v.generate_fbm(int(seed), SERVE["freq"])
        v.Update()
        v.SetScatterRate(SCENE["albedo"])
        v.SetSky(SCENE["sky"])
        vols.append((v, R, float(rng.uniform(*SERVE["alpha"]))))
    n_req = args.serve_requests
    arrivals = np.cumsum(rng.exponential(1.0 / SERVE["rate"], n_req))
    reqs = []
    for i in range(n_req):
        vi = int(rng.integers(len(vols)))
        v, R, alpha = vols[vi]
        Wq, Hq = SERVE["images"][int(rng.integers(len(SERVE["images"])))]
        r = rng.uniform(*SERVE["radius"])
        d = rng.normal(size=3)
        pos = r * d / np.linalg.norm(d)
        ori, up, right = M.camera_frame(tuple(float(x) for x in pos))
        sc = np.float32(np.tan(np.deg2rad(SCENE["fov"]) / 2))
        L = rng.normal(size=3)
        L = (L / np.linalg.norm(L)).astype(np.float32)
        view = v.make_view((Wq, Hq), ori, (up * sc).astype(np.float32), (right * sc).astype(np.float32), L,
                           SCENE["g"], alpha, seed=i)
        reqs.append((vi, view))
    pool = [torch.empty(1920 * 1080 * 4, dtype=torch.float32, device=f"cuda:{local}") for _ in range(64)]
    srv = M.Server(memory_budget=SERVE["budget"], max_slots=args.serve_slots, precision=M.BF16,
                   slot_pixels=1920 * 1080)
    try:
        # warm-up: one request of each image size (LUT, slot buffers), then
        # one small request per volume (its texture copy for the gather)
        for k, (Wq, Hq) in enumerate(SERVE["images"]):
            v = vols[k][0]
            vw = v.make_view((Wq, Hq), *view_vectors(), light(), SCENE["g"], vols[k][2])
            srv.wait(srv.submit(v, vw, pool[k][:Wq * Hq * 4]))
        for k, (v, _, a) in enumerate(vols):
            vw = v.make_view((64, 64), *view_vectors(), light(), SCENE["g"], a)
            srv.wait(srv.submit(v, vw, pool[k % len(pool)][:64 * 64 * 4]))
        tickets = [None] * n_req
        done = [False] * n_req
        t_start = time.perf_counter()

        def producer():
            for i, (vi, view) in enumerate(reqs):
                dt = t_start + arrivals[i] - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                if i >= len(pool):   # buffer reuse: request i - 64 must be done
                    while not done[i - len(pool)]:
                        time.sleep(1e-4)
                tickets[i] = srv.submit(vols[vi][0], view, pool[i % len(pool)][:view.width * view.height * 4])

        th = threading.Thread(target=producer)
        th.start()
        lat, parts, pix = [], [], 0
        first_submit, last_done = None, None
        for i in range(n_req):
            while tickets[i] is None:
                time.sleep(1e-4)
            _, tm = srv.wait(tickets[i])
            done[i] = True
            lat.append(tm["done_ms"] - tm["submit_ms"])
            parts.append((tm["admit_ms"] - tm["submit_ms"], tm["features_ms"] - tm["admit_ms"],
                          tm["network_ms"] - tm["features_ms"], tm["done_ms"] - tm["network_ms"]))
            first_submit = tm["submit_ms"] if first_submit is None else min(first_submit, tm["submit_ms"])
            last_done = tm["done_ms"] if last_done is None else max(last_done, tm["done_ms"])
            pix += reqs[i][1].width * reqs[i][1].height
        th.join()
        st = srv.stats()
        # a burst: 64 requests submitted at once (the same views), to show the
        # batched network at load; the Poisson stream above rarely has two
        # requests' features ready while the network is idle
        b0 = srv.stats()
        tb = time.perf_counter()
        burst = [srv.submit(vols[vi][0], view, pool[i % len(pool)][:view.width * view.height * 4])
                 for i, (vi, view) in enumerate(reqs[:len(pool)])]
        bpix = sum(view.width * view.height for _, view in reqs[:len(pool)])
        blat = [srv.wait(t)[1] for t in burst]
        burst_s = time.perf_counter() - tb
        b1 = srv.stats()
    finally:
        srv.close()
    span_s = (last_done - first_submit) / 1000.0
    lat = np.asarray(lat)
    pm = np.median(np.asarray(parts), axis=0)
    return {"workload": "16 resident fp16 fBm volumes (128/256/512^3, seeds 10-25, alpha 16-256), Poisson "
                        f"{SERVE['rate']:.0f} req/s, images 256^2/512^2/1024^2/1920x1080, orbit cameras, random "
                        f"lights, BF16 network, 120 GB budget, {args.serve_slots} slots sized for 1920x1080 at open, "
                        "results in device buffers",
            "requests": n_req, "offered_req_s": SERVE["rate"], "achieved_req_s": n_req / span_s,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "frames_per_s_1024eq": pix / (1024 * 1024) / span_s,
            "median_split_ms": {"queue": float(pm[0]), "tr+hit+gather": float(pm[1]), "network": float(pm[2]),
                                "result copy": float(pm[3])},
            "batches": st["batches"], "mean_batch": st["batched_requests"] / max(1, st["batches"]),
            "max_batch": st["max_batch"], "peak_bytes": st["peak_bytes"],
            "burst": {"requests": len(burst), "seconds": burst_s, "req_s": len(burst) / burst_s,
                      "frames_per_s_1024eq": bpix / (1024 * 1024) / burst_s,
                      "p50_ms": float(np.percentile([t["done_ms"] - t["submit_ms"] for t in blat], 50)),
                      "batches": b1["batches"] - b0["batches"],
                      "mean_batch": (b1["batched_requests"] - b0["batched_requests"]) /
                                    max(1, b1["batches"] - b0["batches"])}}


def lum_rmse_x100(a, b):
    """The reference's tools/Compare.py metric: both images saturated to 8 bit,
    Rec.601 luminance / 255, RMSE over all pixels, x100."""
    def lum(x):
        q = np.round(np.clip(x[..., :3], 0.0, 1.0) * 255.0)
        return (q[..., 0] * 0.299 + q[..., 1] * 0.587 + q[..., 2] * 0.114) / 255.0
    return float(np.sqrt(np.mean((lum(a) - lum(b)) ** 2)) * 100.0)


def run_precision(args, vol, local):
    """Error of each precision form against the path tracer: the C2 scene seen
    through the headline camera (rendered at 512^2) and through a 1920x1080
    camera (rendered at 480x270, same 16:9 framing).  Reference: one PT launch
    of 4096 spp per pixel, FP64-accumulated, unbiased NEE (one ratio-tracking
    Tr() estimate per vertex), <= 512 bounces.  Predictor: MRPNN running mean
    over 1 and 16 launches."""
    import mrpnn_b200 as M
    ori, up, right = view_vectors()
    views = {"headline camera @512x512": ((512, 512), up, right),
             "1920x1080 camera @480x270": ((480, 270), up, (right * np.float32(16.0 / 9.0)).astype(np.float32))}
    out = {"reference": f"PT, {args.rmse_spp} spp in one launch (FP64 per-pixel sums), unbiased NEE, <= 512 bounces",
           "metrics": "rel_rmse = RMS(pred - PT) / RMS(PT) over linear RGB; lum_rmse_x100 = tools/Compare.py",
           "views": {}}
    prec = {"fp32": M.FP32, "bf16": M.BF16, "fp8": M.FP8}
    L = light()
    for name, (size, u, r) in views.items():
        vol.SetNeeMode(True)
        t0 = time.perf_counter()
        ref = vol.Render(size, ori, u, r, L, M.VolumeRender.PT, SCENE["g"], SCENE["alpha"], multiScatter=512,
                         sampleNum=1, spp=args.rmse_spp, seed=99)
        pt_s = time.perf_counter() - t0
        vol.SetNeeMode(False)
        den = float(np.sqrt(np.mean(ref[..., :3].astype(np.float64) ** 2)))
        res = {"pt_seconds": pt_s}
        for pname, pv in prec.items():
            vol.SetPrecision(pv)
            for n in (1, 16):
                img = vol.Render(size, ori, u, r, L, M.VolumeRender.MRPNN, SCENE["g"], SCENE["alpha"], sampleNum=n,
                                 seed=5)
                d = img[..., :3].astype(np.float64) - ref[..., :3]
                res[f"{pname}_x{n}"] = {"rel_rmse": float(np.sqrt(np.mean(d ** 2)) / den),
                                        "lum_rmse_x100": lum_rmse_x100(img, ref)}
        out["views"][name] = res
    vol.SetPrecision(prec[args.precision])
    return out


LARGE = dict(res=1024, seed=2, freq=8.0, alpha=512.0, albedo=0.999, views=64, size=512, judged=4, judge_size=256,
             judge_spp=1024, radius=(0.8, 2.0))


def run_large(args, local):
    """Large high-order scattering: 1024^3 fBm (seed 2, freq 8), extinction
    512, albedo 0.999, g 0.857; a batch of 64 random orbit views at 512^2 in
    one mrp_render_views call (one FP8 network launch for all views); 4 of
    the views judged against a 1024-spp path-traced image (baked NEE as the
    reference renders, <= 512 bounces), both at 256^2."""
    import torch

    import mrpnn_b200 as M
    t0 = time.perf_counter()
    vol = M.VolumeRender(LARGE["res"], storage="fp16")   # fp16 density grid (2 GiB)
    vol.generate_fbm(LARGE["seed"], LARGE["freq"])
    vol.Update()
    vol.SetScatterRate(LARGE["albedo"])
    vol.SetSky(SCENE["sky"])
    setup_s = time.perf_counter() - t0
    rng = np.random.default_rng(77)
    L = light()
    sc = np.float32(np.tan(np.deg2rad(SCENE["fov"]) / 2))
    cams = []
    for k in range(LARGE["views"]):
        d = rng.normal(size=3)
        pos = rng.uniform(*LARGE["radius"]) * d / np.linalg.norm(d)
        ori, up, right = M.camera_frame(tuple(float(x) for x in pos))
        cams.append((ori, (up * sc).astype(np.float32), (right * sc).astype(np.float32)))
    n = LARGE["size"]
    views = [vol.make_view((n, n), o, u, r, L, SCENE["g"], LARGE["alpha"], seed=k) for k, (o, u, r) in enumerate(cams)]
    outs = [torch.empty((n, n, 4), dtype=torch.float32, device=f"cuda:{local}") for _ in views]
    res = {"workload": f"{LARGE['res']}^3 fp16 fBm (seed 2, freq 8), alpha {LARGE['alpha']:.0f}, albedo {LARGE['albedo']}, "
                       f"g {SCENE['g']}, {LARGE['views']} random orbit views at {n}^2 per mrp_render_views call "
                       "(one batched network launch)", "setup_s": setup_s}
    for pname, pv in (("fp8", M.FP8), ("bf16", M.BF16), ("fp32", M.FP32)):
        vol.SetPrecision(pv)
        vol.render_views(views, outs)
        ms, st = [], []
        for _ in range(3):
            vol.render_views(views, outs)
            ms.append(vol.last_render_ms())
            st.append(vol.last_render_stages())
        t = float(np.median(ms))
        stg = np.median(np.asarray(st), axis=0)
        res[pname] = {"ms_per_batch": t, "views_per_s": LARGE["views"] / (t / 1000.0),
                      "pixels_per_s": LARGE["views"] * n * n / (t / 1000.0),
                      "stage_ms": {"hit + gather (all views)": float(stg[0]), "network (one launch)": float(stg[1]),
                                   "copies": float(stg[2])}}
    # judged views
    if args.large_judge:
        vol.SetBakeResolution(768)
        t1 = time.perf_counter()
        vol.Update_CachedTR(L, LARGE["alpha"])
        bake_s = time.perf_counter() - t1
        m = LARGE["judge_size"]
        judged = {"reference": f"PT {LARGE['judge_spp']} spp (FP64 per-pixel sums), baked 768^3 NEE, <= 512 bounces, "
                               f"{m}^2", "bake_s": bake_s, "views": []}
        for k in range(LARGE["judged"]):
            o, u, r = cams[k]
            t1 = time.perf_counter()
            ref = vol.Render((m, m), o, u, r, L, M.VolumeRender.PT, SCENE["g"], LARGE["alpha"], multiScatter=512,
                             sampleNum=1, spp=LARGE["judge_spp"], seed=500 + k)
            pt_s = time.perf_counter() - t1
            den = float(np.sqrt(np.mean(ref[..., :3].astype(np.float64) ** 2)))
            one = {"pt_seconds": pt_s}
            for pname, pv in (("fp32", M.FP32), ("fp8", M.FP8)):
                vol.SetPrecision(pv)
                img = vol.Render((m, m), o, u, r, L, M.VolumeRender.MRPNN, SCENE["g"], LARGE["alpha"], sampleNum=16,
                                 seed=k)
                dd = img[..., :3].astype(np.float64) - ref[..., :3]
                one[pname] = {"rel_rmse": float(np.sqrt(np.mean(dd ** 2)) / den),
                              "lum_rmse_x100": lum_rmse_x100(img, ref)}
            judged["views"].append(one)
        res["judged"] = judged
    vol.close()
    return res


STAGES = ("first hit + bases", "stencil gather", "network")
# Algorithmic HBM bytes per hit pixel of each predictor stage (fp32 data):
#   gather : 192 points x (8 density + 8 TR + 2 x 4 LUT texels) x 4 B read,
#            576 features x 4 B written
#   network: 576 features x 4 B read + 16 B record + 16 B result
FLOP_PER_HIT = 97072   # 2 x 48,536 MACs of RadiancePredictInternal, grey albedo
# features are fp32 for the FP32 network and FP16 pairs for the tensor-core ones
def stage_bytes_per_hit(precision):
    fb = 4 if precision == "fp32" else 2
    return (None, GATHER_BYTES_PER_PIXEL + 576 * fb, 576 * fb + 32)


def time_frames(vol, view, steps, flush, dev_out, frame0):
    import torch

    import mrpnn_b200 as M
    ms, stages = [], []
    for k in range(steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        view.frame_offset = frame0 + k
        vol.render_view(view, M.VolumeRender.MRPNN, 1, dev_out)
        ms.append(vol.last_render_ms())
        stages.append(vol.last_render_stages())
    return ms, np.mean(np.asarray(stages), axis=0)


def e2e_loops(vol, view, n, host_out, world):
    """Frames/s end to end through the public API, every frame copied to a
    pinned host buffer: mrp_render (each call returns with its frame on the
    host), then the frame loop of mrp_render_start / mrp_render_wait(keep=1),
    in which frame k - 1's copy back overlaps frame k's kernels (two host
    buffers alternate).  Both after three warm-up frames of each API."""
    import mrpnn_b200 as M
    for k in range(3):
        vol.render_view(view, M.VolumeRender.MRPNN, 1, host_out[0])
        vol.render_view_start(view, M.VolumeRender.MRPNN, 1, host_out[k % 2])
    vol.render_wait()
    barrier(world)
    t0 = time.perf_counter()
    for k in range(n):
        view.frame_offset = 2000 + k
        vol.render_view(view, M.VolumeRender.MRPNN, 1, host_out[0])
    sync = n * world / max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    t0 = time.perf_counter()
    for k in range(n):
        view.frame_offset = 3000 + k
        vol.render_view_start(view, M.VolumeRender.MRPNN, 1, host_out[k % 2])
        if k:
            vol.render_wait(keep=1)   # frame k - 1 is in host_out[(k - 1) % 2]
    vol.render_wait()
    return sync, n * world / max_over_ranks(time.perf_counter() - t0, world)


def run_mine(args, rank, world, local):
    import torch

    import mrpnn_b200 as M
    M.init(local)
    precs = {"fp32": M.FP32, "bf16": M.BF16, "fp8": M.FP8}
    vol = M.VolumeRender(RES, storage=args.storage)
    vol.generate_fbm(SCENE["seed"], SCENE["freq"], SCENE["octaves"], SCENE["gain"])
    vol.Update()
    vol.SetScatterRate(SCENE["albedo"])
    vol.SetSky(SCENE["sky"])
    ori, up, right = view_vectors()
    L = light()
    view = vol.make_view((W, H), ori, up, right, L, SCENE["g"], SCENE["alpha"], seed=rank)
    dev_out = torch.empty((H, W, 4), dtype=torch.float32, device=f"cuda:{local}")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")   # > L2 (126 MB)

    # every precision form, same protocol; the headline is args.precision
    others = ("fp32", "bf16", "fp8") if args.all_forms else ()
    order = [p for p in others if p != args.precision] + [args.precision]
    forms = {}
    for p in order:
        vol.SetPrecision(precs[p])
        for i in range(args.warmup):
            view.frame_offset = i
            vol.render_view(view, M.VolumeRender.MRPNN, 1, dev_out)
        torch.cuda.synchronize()
        barrier(world)
        if p == args.precision:
            with ClockSampler(local) as clocks:
                time.sleep(0.3)
                ms, stage_ms = time_frames(vol, view, args.steps, flush, dev_out, 1000)
        else:
            ms, stage_ms = time_frames(vol, view, max(3, args.steps // 4), flush, dev_out, 1000)
        torch.cuda.synchronize()
        barrier(world)
        tot = max_over_ranks(float(sum(ms)), world)
        forms[p] = {"value": len(ms) * world / (tot / 1000.0), "ms_per_frame": tot / len(ms),
                    "stage_ms": dict(zip(STAGES, [round(float(x), 4) for x in stage_ms]))}
    head = forms[args.precision]
    total_ms = head["ms_per_frame"] * args.steps
    value = head["value"]
    img = dev_out.cpu().numpy()
    active = int((img[..., 3] > 0).sum())

    # -- end to end through the public API, every frame to a pinned host buffer:
    # mrp_render (each call returns with its frame on the host), and the
    # frame loop of mrp_render_start / mrp_render_wait(keep=1), in which
    # frame k - 1 is on the host while frame k computes (its copy back
    # overlapped frame k's kernels); two host buffers alternate
    host_out = [torch.empty((H, W, 4), dtype=torch.float32).pin_memory().numpy() for _ in range(2)]
    n_e2e = max(args.e2e_frames, args.steps)
    e2e_sync, e2e = e2e_loops(vol, view, n_e2e, host_out, world)
    # the FP32 drop-in through the same public API (like-for-like with the
    # reference arm, whose MLP is FP32)
    if "fp32" in forms and args.precision != "fp32":
        n_fp32 = max(50, n_e2e // 4)
        vol.SetPrecision(M.FP32)
        fp32_sync, fp32_async = e2e_loops(vol, view, n_fp32, host_out, world)
        vol.SetPrecision(precs[args.precision])
        forms["fp32"]["e2e"] = {"value": fp32_async, "sync_value": fp32_sync, "frames": n_fp32}

    hbm, bf16, peak_kind = peaks()
    st = list(head["stage_ms"].values())
    dom = int(np.argmax(st))
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            traffic = json.load(f).get(f"{args.precision}_{W}x{H}", {}).get(["hit", "gather", "network"][dom])
    except Exception:
        pass
    if dom == 2 and args.precision != "fp32":
        # the tcgen05 network: a GEMM chain, roofline = dense BF16 tensor peak
        flop = active * FLOP_PER_HIT
        achieved = flop / (st[dom] / 1000.0) / 1e12
        dram = (traffic / (st[dom] / 1000.0) / 1e9) if traffic else None
        roof = {"bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s", "frac": achieved / bf16,
                "traffic": traffic, "kernel": STAGES[dom],
                "note": f"algorithmic FLOP = {FLOP_PER_HIT} x {active} hit pixels per launch (grey albedo); "
                        f"duration = CUDA events around the stage; peak {peak_kind} burst bf16 "
                        f"(MEASURED_PEAKS.json bf16_tflops); DRAM from the ncu traffic "
                        f"{'%.0f GB/s' % dram if dram else 'n/a'} of {hbm:.0f}"}
    elif stage_bytes_per_hit(args.precision)[dom] is not None:
        # the gather: its texel reads hit L1 (~80 %), so its roofline is the
        # measured rate of cached loads; HBM is reported beside it
        alg = active * stage_bytes_per_hit(args.precision)[dom]
        achieved = alg / (st[dom] / 1000.0) / 1e9
        dram = traffic / (st[dom] / 1000.0) / 1e9 if traffic else None
        l1 = M.api.measure_l1_rate()
        roof = {"bound": "l1", "achieved": achieved, "peak": l1, "unit": "GB/s", "frac": achieved / l1,
                "traffic": traffic, "kernel": STAGES[dom],
                "hbm": {"peak": hbm, "peak_kind": peak_kind, "algorithmic_frac": achieved / hbm,
                        "dram_achieved": dram, "dram_frac": dram / hbm if dram else None},
                "note": f"algorithmic bytes = {stage_bytes_per_hit(args.precision)[dom]} B x {active} hit pixels per "
                        f"launch (every texel the stencil's trilinear and bilinear fetches read, plus the features "
                        f"written); duration = CUDA events around the stage; peak = the measured rate of cached "
                        f"8-byte loads on this GPU (mrp_measure_l1_rate), since the texel reads are L1 hits.  "
                        f"traffic is the ncu DRAM bytes per launch and hbm.dram_frac what DRAM carries; the kernel "
                        f"is issue-bound (profiles/k_gather_rec_512x512.md)"}
    else:
        roof = {"bound": "hbm", "achieved": None, "peak": hbm, "unit": "GB/s", "frac": None, "traffic": traffic,
                "kernel": STAGES[dom], "note": "march lookups are data dependent; see profiles/"}
    if dom == 2 and args.precision == "fp32":
        # the FP32 drop-in network: SIMT FMAs, roofline = the CUDA cores' FP32
        # rate (no measured figure exists for it: nominal 128 FMA lanes per SM)
        flop = active * FLOP_PER_HIT
        achieved = flop / (st[dom] / 1000.0) / 1e12
        mhz = clocks.summary().get("sm_max_mhz") or 1965.0
        fp32_peak = torch.cuda.get_device_properties(local).multi_processor_count * 128 * 2 * mhz * 1e6 / 1e12
        roof = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "traffic": traffic, "kernel": STAGES[dom],
                "note": f"algorithmic FLOP = {FLOP_PER_HIT} x {active} hit pixels per launch; duration = CUDA events "
                        f"around the stage; peak = nominal FP32 FMA rate of the SMs at {mhz:.0f} MHz (not measured)"}

    tracer = run_tracer(args, local) if (rank == 0 and args.tracer_steps > 0) else None
    serving = run_serving(args, local) if (rank == 0 and args.serve_requests > 0) else None
    precision_error = run_precision(args, vol, local) if (rank == 0 and args.rmse_spp > 0) else None
    large = run_large(args, local) if (rank == 0 and args.large) else None

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sc = cpu_scene_from_gpu(vol)
        n_cpu = min(args.cpu_pixels, W * H)
        pix_s, dt, px, ref = time_cpu_predict(sc, n_cpu, reps=args.cpu_reps, want=True)
        cpu = {"value": pix_s / (W * H), "unit": UNIT, "cores": omp_threads(), "kind": "port",
               "sample": f"{args.cpu_reps} passes over {n_cpu} pixels of the {W}x{H} frame ({dt:.1f} s), "
                         f"OpenMP oracle (first hit, gather, FP32 MLP)"}
        parity = frame_parity(vol, px, ref, local)
        cpu["torch_network"] = time_torch_network(sc, active)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp32": "f32", "bf16": "bf16", "fp8": "fp8-e4m3"}[args.precision], "data": "synthetic",
            "config": {"workload": f"MRPNN predictor frame {W}x{H}, {RES}^3 fBm cloud (seed 1, freq 6), 9-level pyramid",
                       "precision": args.precision, "grid_storage": args.storage, "parallelism": f"replicas x{world}",
                       "l2": "flushed (256 MiB write) between timed steps", "hit_pixels": active,
                       "precision_forms": forms},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 96, "d2h_bytes_per_step": W * H * 16,
                    "frames": n_e2e,
                    "api": "mrp_render_start + mrp_render_wait(keep=1) frame loop, pinned host buffers",
                    "sync_value": e2e_sync, "sync_api": "mrp_render per frame, pinned host buffer"},
            "gpu_launches": args.steps * 3,
            "roofline": roof,
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": clocks.summary(),
            "tracer": tracer,
            "serving": serving,
            "precision_error": precision_error,
            "large": large,
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--precision", default="bf16", choices=["fp32", "bf16", "fp8"])
    ap.add_argument("--cpu-pixels", type=int, default=1 << 20,
                    help="pixels of the CPU-baseline sample (default: the full 1024^2 frame)")
    ap.add_argument("--cpu-reps", type=int, default=3, help="passes over the CPU-baseline sample (~10 s on 16 cores)")
    ap.add_argument("--ref-pixels", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--size", type=int, default=1024, help="frame edge (the headline workload is 1024)")
    ap.add_argument("--storage", default="fp32", choices=["fp32", "fp16"],
                    help="density grid storage of the headline volume (fp32: the reference's float grid)")
    ap.add_argument("--tracer-steps", type=int, default=3, help="timed PT frames of the tracer workload (0: skip)")
    ap.add_argument("--tracer-cpu-frames", type=int, default=20,
                    help="whole frames of the tracer's CPU baseline (0: skip)")
    ap.add_argument("--e2e-frames", type=int, default=200, help="frames of each end-to-end loop (at least --steps)")
    ap.add_argument("--all-forms", type=int, default=1,
                    help="also time the other precision forms (0: the headline form only, e.g. for profiling)")
    ap.add_argument("--serve-requests", type=int, default=400, help="requests of the serving workload (0: skip)")
    ap.add_argument("--serve-slots", type=int, default=SERVE["slots"], help="request slots of the server")
    ap.add_argument("--rmse-spp", type=int, default=4096, help="spp of the PT reference image (0: skip)")
    ap.add_argument("--large", type=int, default=1, help="run the 1024^3 / 64-view workload (0: skip)")
    ap.add_argument("--large-judge", type=int, default=1, help="judge 4 large views against the tracer (0: skip)")
    args = ap.parse_args()
    global W, H
    W = H = args.size
    rank, world, local = (0, 1, 0)
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", 0))
        world = int(os.environ.get("WORLD_SIZE", 1))
        run_reference(args, rank, world)
        return
    rank, world, local = dist_setup(args.gpus)
    try:
        run_mine(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
