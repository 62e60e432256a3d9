"""Generate tests/golden/ref_pins.npz from the reference's own render code.

The reference's core/vector.cu, core/radiancePredict.cu,
core/renderResources.cu and core/render.cuh are compiled on the CPU by
oracle/Makefile ("make -C oracle ref", shims in oracle/ref/shim) into
oracle/_ref/libmrpnn_ref.so.  This script feeds it seeded inputs and stores
inputs and outputs, so tests can pin the oracle (oracle/mrpnn_oracle.cpp) to
the reference without the reference tree being present.

Scene-based cases use a small synthetic scene rebuilt identically by the test
(fBm 32^3, pyramid, TR mips, the HG-LUT rows the gather reads); checksums of
those scene arrays are stored too.

Usage: python tests/golden/make_golden.py   (needs the reference tree that
oracle/Makefile reads: its REF default, or MRPNN_REFERENCE)
"""
import ctypes as C
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_pins.npz")

SCENE = dict(R=32, seed=0, freq=4.0, alpha=64.0, g=0.857, lut_seed=7, light=(0.3, 0.8, 0.5),
             sr=(0.99, 0.99, 0.99), sky=(0.05, 0.05, 0.05))


def light_dir():
    L = np.asarray(SCENE["light"], np.float32)
    return (L / np.float32(np.sqrt(np.float32(np.dot(L, L))))).astype(np.float32)


def build_scene():
    """The synthetic scene used by the scene-based pins (oracle-built)."""
    R = SCENE["R"]
    vol = O.fbm_volume(R, SCENE["seed"], SCENE["freq"])
    md = O.lib().orc_max_density(vol, vol.size)
    mips = O.build_pyramid(vol, R)
    L = light_dir()
    tr = O.tr_mips(mips, SCENE["alpha"], L)
    _, tex = O.lut_rows_needed()
    lut = np.zeros(512 * 512, np.float32)
    lut[tex] = O.hg_lut_texels(SCENE["g"], SCENE["lut_seed"], tex)
    baked = tr[:128 ** 3].copy()   # any clamp-sampled grid serves as the NEE table here
    sc = O.SceneBuf(vol, R, md, mips, tr, lut, baked=baked, baked_res=128, scatter_rate=SCENE["sr"],
                    sky=SCENE["sky"])
    return sc


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def camera(W):
    ori = np.array([0.75, 0.75, 0.75], np.float32)
    fwd = -ori / np.float32(np.sqrt(np.float32(np.dot(ori, ori))))
    right = np.cross([0, 1, 0], fwd).astype(np.float32)
    right /= np.float32(np.sqrt(np.float32(np.dot(right, right))))
    up = np.cross(fwd, right).astype(np.float32)
    t = np.float32(np.tan(np.deg2rad(22.5)))
    return ori, (up * t).astype(np.float32), (right * t).astype(np.float32)


def smooth_lut():
    """A smooth 512 x 512 table (rows: cone angle, columns: cos theta) for the
    GetHGLut pins, rebuilt identically by the tests."""
    j, i = np.mgrid[0:512, 0:512].astype(np.float32)
    return (np.float32(1.5) + np.sin(i * np.float32(0.021)) * np.cos(j * np.float32(0.013))).astype(np.float32)


def lut_queries(rng, n=256):
    """(cos, angle) queries for GetHGLut, the table's edges included."""
    c = rng.uniform(-1.05, 1.05, n).astype(np.float32)
    a = rng.uniform(-0.05, 1.1, n).astype(np.float32)
    c[:6] = [-1.0, 1.0, 0.0, -1.0, 1.0, 0.5]
    a[:6] = [0.0, 0.0, 0.0, 1.0471975, 1.0471975, 0.5]
    return np.stack([c, a], 1)


BAKE_RES = 48
HDRI_ENV_EXP = 1.7


def smooth_hdri(w=48, h=24):
    """A smooth synthetic equirect map, float32 [h, w, 4], rebuilt
    identically by the tests (bright band near the horizon, warm to cold)."""
    j, i = np.mgrid[0:h, 0:w].astype(np.float32)
    band = np.exp(-((j - np.float32(h * 0.45)) / np.float32(h * 0.2)) ** 2).astype(np.float32)
    r = np.float32(0.2) + band * (np.float32(1.0) + np.float32(0.5) * np.sin(i * np.float32(0.26)))
    g = np.float32(0.3) + np.float32(0.6) * band
    b = np.float32(0.9) - np.float32(0.5) * band + np.float32(0.05) * np.cos(j * np.float32(0.7))
    return np.stack([r, g, b, np.ones_like(r)], -1).astype(np.float32)


def hdri_pins(out, rng):
    """NNPredict and CalculateRadiance with an environment map bound
    (SkyBox, core/render.cuh:24-27): missed pixels and escaping paths."""
    R = O.ref()
    sc = build_scene()
    sc2 = O.SceneBuf(sc.density, sc.res, sc.max_density, sc.mips, sc.tr, sc.lut, baked=sc.baked,
                     baked_res=sc.baked_res, scatter_rate=SCENE["sr"], sky=SCENE["sky"], hdri=smooth_hdri(),
                     env_exp=HDRI_ENV_EXP)
    sc2.bind_ref()
    L = light_dir()
    W = 16
    ori, up, right = camera(W)
    up, right = (up * np.float32(2.5)).astype(np.float32), (right * np.float32(2.5)).astype(np.float32)
    px = np.arange(W * W, dtype=np.int32)
    rgba = np.zeros((W * W, 4), np.float32)
    R.ref_predict_pixels(W, W, ori, up, right, L, np.ones(3, np.float32), SCENE["alpha"], SCENE["g"], 5, 2, px,
                         W * W, rgba)
    out["hdri_pp_rgba"] = rgba
    cases = [(int(p_), int(k_)) for p_, k_ in zip(rng.integers(0, W * W, 48), rng.integers(0, 8, 48))]
    tr_out = np.zeros((len(cases), 4), np.float32)
    for i, (p_, k_) in enumerate(cases):
        o4 = np.zeros(4, np.float32)
        R.ref_trace_sample(W, W, ori, up, right, L, np.ones(3, np.float32), SCENE["alpha"], SCENE["g"], 64, 5, 2,
                           p_, k_, o4)
        tr_out[i] = o4
    out["hdri_ts_cases"], out["hdri_ts_out"] = np.asarray(cases, np.int32), tr_out
    sc.bind_ref()


def volume_pins(out, rng):
    """VolumeRender::Update's pyramid, Update_TR (device and host branches),
    Fill_Hg texels, GetHGLut and Fill_BakeTR voxels from the reference's
    core/volume.cu compiled on the CPU (oracle/_ref/libmrpnn_ref_volume.so)."""
    R = SCENE["R"]
    vol = O.fbm_volume(R, SCENE["seed"], SCENE["freq"])
    L = light_dir()
    out["vol_pyramid_digest"] = np.array(digest(O.ref_pyramid(vol, R)))
    v300 = O.fbm_volume(300, 3, 5.0)
    out["vol_pyramid300_digest"] = np.array(digest(O.ref_pyramid(v300, 300)))
    out["vol_tr_digest"] = np.array(digest(O.ref_tr(vol, R, SCENE["alpha"], L, cpu=False)))
    out["vol_tr_cpu_digest"] = np.array(digest(O.ref_tr(vol, R, SCENE["alpha"], L, cpu=True)))
    tex = np.sort(rng.choice(512 * 512, 256, replace=False)).astype(np.int32)
    out["vol_lut_texels"] = tex
    for tag, g in LUT_GS:
        out[f"vol_lut_{tag}"] = O.ref_hg_texels(g, SCENE["lut_seed"], tex)
    q = lut_queries(rng)
    lut = smooth_lut()
    out["vol_getlut_q"] = q
    out["vol_getlut_out"] = np.array([O.ref_get_hg_lut(lut, c, a) for c, a in q], np.float32)
    md = O.lib().orc_max_density(vol, vol.size)
    vox = np.sort(rng.choice(BAKE_RES ** 3, 512, replace=False)).astype(np.int64)
    out["vol_bake_vox"] = vox
    out["vol_bake_out"] = O.ref_bake_voxels(vol, R, md, SCENE["alpha"], L, BAKE_RES, SCENE["lut_seed"], vox)


LUT_GS = (("g0857", 0.857), ("gm05", -0.5), ("g065", 0.65))

VIEWER = dict(W=24, H=24, multi=32, seed=5, frame=2, exposure=1.3)
FINISH_MODES = ((0, 0, 2), (0, 1, 1), (1, 0, 2), (0, 1, 0))   # (predict, denoise, tone)


def viewer_pins(out, rng):
    """The viewer frame: RenderCamera<false> with the histogram buffer over
    two frames (checkerboard, flip 1; square: the reference bounds pixels by
    the opposite edges, core/volume.cu:102), then the finishing pass in each mode
    (Denoise / ReprojectionDenoise, Gamma / ACES / none, RGBA8), from
    core/volume.cu compiled on the CPU."""
    sc = build_scene()
    V = VIEWER
    W, H = V["W"], V["H"]
    ori, up, right = camera(W)
    L = light_dir()
    tgt = rng.uniform(0, 1, W * H * 3).astype(np.float32)
    his = rng.uniform(0, 2, W * H * 33).astype(np.float32)
    out["vw_target0"], out["vw_histo0"] = tgt.copy(), his.copy()
    for fnum in (0, 1):
        O.ref_volume().ref_vol_frame_pt(sc.density, sc.res, sc.max_density, sc.baked, sc.baked_res, sc.scatter_rate,
                                        sc.sky, W, H, ori, up, right, L, np.ones(3, np.float32), SCENE["alpha"],
                                        SCENE["g"], V["multi"], V["seed"], V["frame"] + fnum, 2 * fnum, 1, 1, tgt, his)
    out["vw_target"], out["vw_histo"] = tgt, his
    for k, (pred, den, tone) in enumerate(FINISH_MODES):
        for fn in (0, 5):
            o8 = np.zeros(W * H, np.uint32)
            h = his.copy()
            O.ref_volume().ref_vol_frame_finish(tgt.copy(), h, W, H, fn, 1, pred, den, V["exposure"], tone, o8)
            out[f"vw_rgba8_{k}_{fn}"] = o8
            out[f"vw_histo_{k}_{fn}"] = h


def main():
    R = O.ref()
    rng = np.random.default_rng(20261203)
    out = {}

    # -- MLP (RadiancePredictInternal) on random features ---------------------
    n = 64
    feat = rng.uniform(0.0, 1.5, (n, 576)).astype(np.float32)
    gam = rng.uniform(0.0, np.pi, n).astype(np.float32)
    out["mlp_feat"], out["mlp_gamma"] = feat, gam
    for tag, sr in (("grey", (1.0, 1.0, 1.0)), ("rgb", (0.99, 0.9, 0.8))):
        out[f"mlp_out_{tag}"] = O.ref_mlp(feat, gam, 0.857, sr)
        out[f"mlp_sr_{tag}"] = np.asarray(sr, np.float32)

    # -- stencil tables (GetSamples23_, SphereRandom3) ------------------------
    offs, layers, types, lidx, dirs = [], [], [], [], []
    for i in range(192):
        o, l, t, li = C.c_float(), C.c_float(), C.c_int(), C.c_int()
        d = np.zeros(3, np.float32)
        R.ref_stencil(i, C.byref(o), C.byref(l), C.byref(t), C.byref(li), d)
        offs.append(o.value); layers.append(l.value); types.append(t.value); lidx.append(li.value); dirs.append(d)
    out["st_offset"] = np.asarray(offs, np.float32)
    out["st_layer"] = np.asarray(layers, np.float32)
    out["st_type"] = np.asarray(types, np.int32)
    out["st_localindex"] = np.asarray(lidx, np.int32)
    out["st_dirs"] = np.asarray(dirs, np.float32)

    # -- maths -------------------------------------------------------------------
    m = 512
    hc = rng.uniform(-1, 1, m).astype(np.float32)
    hgv = rng.uniform(-0.95, 0.95, m).astype(np.float32)
    out["hg_in"] = np.stack([hc, hgv], 1)
    out["hg_out"] = np.array([R.ref_hg(c, g) for c, g in zip(hc, hgv)], np.float32)
    e = rng.uniform(0, 1, (m, 2)).astype(np.float32)
    vv = rng.normal(size=(m, 3)).astype(np.float32)
    vv /= np.linalg.norm(vv, axis=1, keepdims=True).astype(np.float32)
    out["shg_e"], out["shg_v"], out["shg_g"] = e, vv, hgv
    res = np.zeros((m, 3), np.float32)
    for i in range(m):
        o3 = np.zeros(3, np.float32)
        R.ref_sample_hg(e[i, 0], e[i, 1], np.ascontiguousarray(vv[i]), hgv[i], o3)
        res[i] = o3
    out["shg_out"] = res
    p = rng.uniform(-1.2, 1.2, (m, 3)).astype(np.float32)
    d = rng.normal(size=(m, 3)).astype(np.float32)
    d[rng.uniform(size=m) < 0.1, rng.integers(0, 3)] = 0.0
    out["rb_p"], out["rb_d"] = p, d
    out["rb_off"] = np.array([R.ref_ray_box_offset(p[i], d[i]) for i in range(m)], np.float32)
    out["rb_dist"] = np.array([R.ref_ray_box_distance(p[i], d[i]) for i in range(m)], np.float32)

    # -- scene-based pins ----------------------------------------------------------
    sc = build_scene()
    sc.bind_ref()
    out["scene_digest_mips"] = np.array(digest(sc.mips))
    out["scene_digest_tr"] = np.array(digest(sc.tr))
    out["scene_digest_lut"] = np.array(digest(sc.lut))
    L = light_dir()
    # first hit
    k = 256
    oris = (np.array([0.75, 0.75, 0.75]) + rng.normal(0, 0.05, (k, 3))).astype(np.float32)
    dirs_ = (-oris + rng.normal(0, 0.2, (k, 3))).astype(np.float32)
    hits = np.zeros((k, 4), np.float32)
    for i in range(k):
        h = np.zeros(3, np.float32)
        a = R.ref_first_hit(oris[i], dirs_[i], SCENE["alpha"], h)
        hits[i, :3], hits[i, 3] = h, a
    out["fh_ori"], out["fh_dir"], out["fh_out"] = oris, dirs_, hits
    # basis (GetMatrixFromNormal)
    k = 64
    bv = rng.normal(size=(k, 3)).astype(np.float32)
    bo = np.zeros((k, 9), np.float32)
    for i in range(k):
        o9 = np.zeros(9, np.float32)
        R.ref_basis(bv[i], 0.1, i, 0, 3, 11, 0, o9)
        bo[i] = o9
    out["basis_v"], out["basis_out"] = bv, bo
    # SetupInputData
    k = 32
    pos = rng.uniform(-0.45, 0.45, (k, 3)).astype(np.float32)
    bases = np.zeros((k, 12), np.float32)
    feats = np.zeros((k, 576), np.float32)
    gams = np.zeros(k, np.float32)
    for i in range(k):
        m9 = np.zeros(9, np.float32)
        l9 = np.zeros(9, np.float32)
        R.ref_basis(rng.normal(size=3).astype(np.float32), 0.1, i, 0, 0, 0, 0, m9)
        R.ref_basis(L, 0.1, i, 1, 0, 0, 0, l9)
        bases[i, :9], bases[i, 9:] = m9, l9[:3]
        f = np.zeros(576, np.float32)
        gm = np.zeros(1, np.float32)
        R.ref_setup_input(1, pos[i], m9[:3], m9[3:6], m9[6:], l9[:3], L, SCENE["g"], SCENE["alpha"], f, gm)
        feats[i], gams[i] = f, gm[0]
    out["si_pos"], out["si_bases"], out["si_feat"], out["si_gamma"] = pos, bases, feats, gams
    # full predictor pixels (RenderCamera<true, MRPNN> ray + NNPredict<MRPNN>)
    W = 16
    ori, up, right = camera(W)
    px = np.arange(W * W, dtype=np.int32)
    rgba = np.zeros((W * W, 4), np.float32)
    R.ref_predict_pixels(W, W, ori, up, right, L, np.ones(3, np.float32), SCENE["alpha"], SCENE["g"], 5, 2, px,
                         W * W, rgba)
    out["pp_rgba"] = rgba
    # tracer samples (CalculateRadiance, one sample per call)
    cases = [(int(p_), int(k_)) for p_, k_ in zip(rng.integers(0, W * W, 48), rng.integers(0, 8, 48))]
    tr_out = np.zeros((len(cases), 4), np.float32)
    for i, (p_, k_) in enumerate(cases):
        o4 = np.zeros(4, np.float32)
        R.ref_trace_sample(W, W, ori, up, right, L, np.ones(3, np.float32), SCENE["alpha"], SCENE["g"], 64, 5, 2,
                           p_, k_, o4)
        tr_out[i] = o4
    out["ts_cases"], out["ts_out"] = np.asarray(cases, np.int32), tr_out
    # Tr (ratio + delta tracking)
    k = 64
    tp = rng.uniform(-0.45, 0.45, (k, 3)).astype(np.float32)
    tv = np.zeros(k, np.float32)
    for i in range(k):
        dis = R.ref_ray_box_distance(tp[i], L)
        tv[i] = R.ref_tr(tp[i], L, dis, SCENE["alpha"], i, 0, 0, 9, 2)
    out["tr_pos"], out["tr_out"] = tp, tv

    # tile gather of the tile network (GatherSamples -> NNGatherSamples)
    TW = 6
    tori, tup, tright = camera(TW)
    tiles = np.zeros((TW * TW, 773), np.float32)
    for idx in range(TW * TW):
        o = np.zeros(773, np.float32)
        R.ref_gather_tile(TW, TW, tori, tup, tright, L, SCENE["alpha"], SCENE["g"], 5, 2, 3, 5, idx, o)
        tiles[idx] = o
    out["tile_out"] = tiles

    # -- environment map (SetHDRI / SkyBox) ----------------------------------------
    hdri_pins(out, rng)

    # -- volume builders: core/volume.cu's own code on the CPU --------------------
    volume_pins(out, rng)
    viewer_pins(out, rng)

    np.savez_compressed(OUT, **out)
    print(OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
