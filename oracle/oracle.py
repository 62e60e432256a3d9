"""ctypes loader for the CPU oracle (``libmrpnn_oracle.so``) and for the
reference's own sources compiled on the CPU (``_ref/libmrpnn_ref.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline legs of bench.py, never by the product package.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libmrpnn_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmrpnn_ref.so")
REF_VOLUME_SO = os.path.join(HERE, "_ref", "libmrpnn_ref_volume.so")
# The reference tree is located by oracle/Makefile (its REF variable, which
# MRPNN_REFERENCE overrides); this module never names a path of its own.
REF_TREE_ENV = "MRPNN_REFERENCE"
MODEL = os.path.join(os.path.dirname(HERE), "mrpnn_b200", "data", "mrpnn_model.bin")

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
F3 = C.c_float * 3


class Scene(C.Structure):
    _fields_ = [("density", C.c_void_p), ("res", C.c_int), ("max_density", C.c_float),
                ("mips", C.c_void_p), ("tr_mips", C.c_void_p), ("hg_lut", C.c_void_p),
                ("baked_tr", C.c_void_p), ("baked_res", C.c_int),
                ("scatter_rate", F3), ("tr_scale", C.c_float), ("sky", F3),
                ("hdri", C.c_void_p), ("hdri_w", C.c_int), ("hdri_h", C.c_int), ("env_exp", C.c_float)]


class View(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("ori", F3), ("up", F3), ("right", F3),
                ("light_dir", F3), ("light_color", F3), ("alpha", C.c_float), ("g", C.c_float),
                ("multi_scatter", C.c_int), ("spp", C.c_int), ("seed", C.c_uint32), ("frame", C.c_int)]


def _build(target):
    make = shutil.which("make")
    if make is None:
        raise RuntimeError("oracle library missing and no make to build it")
    subprocess.run([make, "-s", "-C", HERE, target], check=True)


_lib = None
_ref = None
_ref_vol = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            _build("all")
        L = C.CDLL(ORACLE_SO)
        L.orc_load_model.argtypes = [C.c_char_p]
        L.orc_philox4x32_10.argtypes = [np.ctypeslib.ndpointer(np.uint32), np.ctypeslib.ndpointer(np.uint32),
                                        np.ctypeslib.ndpointer(np.uint32)]
        L.orc_stream_uniform.argtypes = [C.c_uint32] * 6
        L.orc_stream_uniform.restype = C.c_float
        L.orc_fbm_voxel.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_float, C.c_int, C.c_float]
        L.orc_fbm_voxel.restype = C.c_float
        L.orc_fbm_volume.argtypes = [f32p, C.c_int, C.c_uint32, C.c_float, C.c_int, C.c_float]
        L.orc_max_density.argtypes = [f32p, C.c_int64]
        L.orc_max_density.restype = C.c_float
        L.orc_build_pyramid.argtypes = [f32p, C.c_int, f32p]
        L.orc_tr_mip_level.argtypes = [f32p, C.c_int, C.c_float, f32p, f32p]
        L.orc_hg_lut_texels.argtypes = [C.c_float, C.c_uint32, i32p, C.c_int, f32p]
        L.orc_baked_tr.argtypes = [C.POINTER(Scene), C.c_float, f32p, C.c_int, C.c_uint32, C.c_int, i64p,
                                   C.c_int64, f32p]
        L.orc_tr.argtypes = [C.POINTER(Scene), f32p, f32p, C.c_float, C.c_float] + [C.c_uint32] * 5
        L.orc_tr.restype = C.c_float
        L.orc_stencil_tables.argtypes = [f32p, i32p, i32p, i32p, f32p]
        L.orc_hg.argtypes = [C.c_float, C.c_float]
        L.orc_hg.restype = C.c_float
        L.orc_sample_hg.argtypes = [C.c_float, C.c_float, f32p, C.c_float, f32p]
        L.orc_ray_box_offset.argtypes = [f32p, f32p]
        L.orc_ray_box_offset.restype = C.c_float
        L.orc_ray_box_distance.argtypes = [f32p, f32p]
        L.orc_ray_box_distance.restype = C.c_float
        L.orc_sample_density.argtypes = [f32p, C.c_int, f32p, C.c_int]
        L.orc_sample_density.restype = C.c_float
        L.orc_sample_lut.argtypes = [f32p, C.c_float, C.c_float]
        L.orc_sample_lut.restype = C.c_float
        L.orc_camera_ray.argtypes = [C.POINTER(View), C.c_int, C.c_int, f32p]
        L.orc_first_hit.argtypes = [C.POINTER(Scene), f32p, f32p, C.c_float, f32p]
        L.orc_basis.argtypes = [f32p, C.c_float, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                C.POINTER(C.c_uint32), f32p]
        L.orc_setup_input.argtypes = [C.POINTER(Scene), C.c_int] + [f32p] * 6 + [C.c_float, C.c_float, f32p, f32p]
        L.orc_mlp_f32.argtypes = [f32p, f32p, C.c_float, f32p, C.c_int, f32p]
        L.orc_mlp_f64.argtypes = [f32p, f32p, C.c_float, f32p, C.c_int, f64p]
        L.orc_predict_pixels.argtypes = [C.POINTER(Scene), C.POINTER(View), i32p, C.c_int, f32p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]
        L.orc_trace_pixels.argtypes = [C.POINTER(Scene), C.POINTER(View), i32p, C.c_int, f32p, C.c_void_p,
                                       C.c_void_p]
        L.orc_frame_pt.argtypes = [C.POINTER(Scene), C.POINTER(View), C.c_int, C.c_int, C.c_int, C.c_void_p,
                                   C.c_void_p]
        L.orc_frame_finish.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_float, C.c_int, C.c_void_p]
        L.orc_gather_tiles.argtypes = [C.POINTER(Scene), C.POINTER(View), C.c_int, C.c_int, C.c_void_p]
        L.orc_trace_rays.argtypes = [C.POINTER(Scene), C.POINTER(View), C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_void_p, C.c_void_p]
        L.orc_get_samples.argtypes = [C.POINTER(Scene)] + [C.c_void_p] * 6 + [C.c_int, F3, C.c_int, C.c_int,
                                                                               C.c_uint32, C.c_void_p]
        L.orc_get_trs.argtypes = [C.POINTER(Scene), C.c_float, C.c_void_p, C.c_void_p, C.c_int, F3, F3, C.c_float,
                                  C.c_int, C.c_uint32, C.c_void_p]
        L.orc_env_light.argtypes = [C.POINTER(Scene), C.c_float, C.c_int, f32p, f32p]
        L.orc_roberts2.argtypes = [C.c_int, f32p]
        L.orc_uniform_sample_sphere.argtypes = [C.c_float, C.c_float, f32p]
        L.orc_image_sample.argtypes = [f32p, C.c_int, C.c_int, C.c_float, C.c_float, f32p]
        rc = L.orc_load_model(MODEL.encode())
        if rc != 0:
            raise RuntimeError(f"oracle: cannot load model file {MODEL} (rc={rc})")
        _lib = L
    return _lib


def _make_ref_args():
    tree = os.environ.get(REF_TREE_ENV)
    return [f"REF={tree}"] if tree else []


def ref_tree():
    """The reference tree the Makefile's `ref` target compiles from."""
    make = shutil.which("make") or "make"
    r = subprocess.run([make, "-s", "-C", HERE, "ref-tree"] + _make_ref_args(), capture_output=True, text=True)
    return r.stdout.strip() if r.returncode == 0 else ""


def ref_available():
    if os.path.exists(REF_SO):
        return True
    tree = ref_tree()
    return bool(tree) and os.path.isdir(os.path.join(tree, "core"))


def ref():
    """The reference's render sources compiled on the CPU (built on demand)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            if not ref_available():
                raise RuntimeError("reference checker not built and reference tree absent")
            subprocess.run([shutil.which("make") or "make", "-s", "-C", HERE, "ref"] + _make_ref_args(), check=True)
        R = C.CDLL(REF_SO)
        vp = C.c_void_p
        R.ref_bind_scene.argtypes = [vp, C.c_int, C.c_float, vp, vp, vp, vp, C.c_int, f32p, C.c_float, f32p,
                                     vp, C.c_int, C.c_int, C.c_float]
        R.ref_hg.argtypes = [C.c_float, C.c_float]
        R.ref_hg.restype = C.c_float
        R.ref_sample_hg.argtypes = [C.c_float, C.c_float, f32p, C.c_float, f32p]
        R.ref_ray_box_offset.argtypes = [f32p, f32p]
        R.ref_ray_box_offset.restype = C.c_float
        R.ref_ray_box_distance.argtypes = [f32p, f32p]
        R.ref_ray_box_distance.restype = C.c_float
        R.ref_stencil.argtypes = [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), f32p]
        R.ref_sample_density.argtypes = [C.c_int, f32p]
        R.ref_sample_density.restype = C.c_float
        R.ref_shadow_tr.argtypes = [f32p, f32p, C.c_int]
        R.ref_shadow_tr.restype = C.c_float
        R.ref_mlp.argtypes = [f32p, f32p, C.c_float, f32p, C.c_int, f32p]
        R.ref_setup_input.argtypes = [C.c_int] + [f32p] * 6 + [C.c_float, C.c_float, f32p, f32p]
        R.ref_first_hit.argtypes = [f32p, f32p, C.c_float, f32p]
        R.ref_basis.argtypes = [f32p, C.c_float] + [C.c_uint32] * 5 + [f32p]
        R.ref_tr.argtypes = [f32p, f32p, C.c_float, C.c_float] + [C.c_uint32] * 5
        R.ref_tr.restype = C.c_float
        R.ref_predict_pixels.argtypes = [C.c_int, C.c_int, f32p, f32p, f32p, f32p, f32p, C.c_float, C.c_float,
                                         C.c_uint32, C.c_int, i32p, C.c_int, f32p]
        R.ref_trace_sample.argtypes = [C.c_int, C.c_int, f32p, f32p, f32p, f32p, f32p, C.c_float, C.c_float,
                                       C.c_int, C.c_uint32, C.c_int, C.c_int, C.c_int, f32p]
        R.ref_gather_tile.argtypes = [C.c_int, C.c_int, f32p, f32p, f32p, f32p, C.c_float, C.c_float, C.c_uint32,
                                      C.c_int, C.c_int, C.c_int, C.c_int, f32p]
        _ref = R
    return _ref


def ref_volume():
    """The reference's core/volume.cu volume builders compiled on the CPU
    (built on demand with the `ref` target)."""
    global _ref_vol
    if _ref_vol is None:
        if not os.path.exists(REF_VOLUME_SO):
            if not ref_available():
                raise RuntimeError("reference checker not built and reference tree absent")
            subprocess.run([shutil.which("make") or "make", "-s", "-C", HERE, "ref"] + _make_ref_args(), check=True)
        R = C.CDLL(REF_VOLUME_SO)
        R.ref_vol_pyramid.argtypes = [f32p, C.c_int, f32p]
        R.ref_vol_tr.argtypes = [f32p, C.c_int, C.c_float, f32p, C.c_int, f32p]
        R.ref_vol_hg_texels.argtypes = [C.c_float, C.c_uint32, i32p, C.c_int, f32p]
        R.ref_vol_get_hg_lut.argtypes = [f32p, C.c_float, C.c_float]
        R.ref_vol_get_hg_lut.restype = C.c_float
        R.ref_vol_bake_voxels.argtypes = [f32p, C.c_int, C.c_float, C.c_float, f32p, C.c_int, C.c_uint32, i64p,
                                          C.c_int, f32p]
        R.ref_vol_load_hdr.argtypes = [C.c_char_p, C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.c_void_p, C.c_size_t]
        R.ref_vol_frame_pt.argtypes = [f32p, C.c_int, C.c_float, f32p, C.c_int, f32p, f32p, C.c_int, C.c_int] + \
            [f32p] * 5 + [C.c_float, C.c_float, C.c_int, C.c_uint32, C.c_int, C.c_int, C.c_int, C.c_int, f32p, f32p]
        R.ref_vol_frame_finish.argtypes = [f32p, f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_float, C.c_int, np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")]
        R.ref_vol_roberts2.argtypes = [C.c_int, f32p]
        R.ref_vol_uniform_sample_sphere.argtypes = [C.c_float, C.c_float, f32p]
        R.ref_vol_image_sample.argtypes = [f32p, C.c_int, C.c_int, C.c_float, C.c_float, f32p]
        _ref_vol = R
    return _ref_vol


def ref_pyramid(data, R):
    out = np.empty(sum(r ** 3 for r in mip_sizes()), np.float32)
    ref_volume().ref_vol_pyramid(np.ascontiguousarray(data, np.float32).ravel(), R, out)
    return out


def ref_tr(data, R, alpha, light_dir, cpu=False):
    out = np.empty(sum(r ** 3 for r in tr_sizes()), np.float32)
    ref_volume().ref_vol_tr(np.ascontiguousarray(data, np.float32).ravel(), R, alpha,
                            np.asarray(light_dir, np.float32), 1 if cpu else 0, out)
    return out


def ref_hg_texels(g, seed, texels):
    t = np.ascontiguousarray(texels, np.int32)
    out = np.empty(t.size, np.float32)
    ref_volume().ref_vol_hg_texels(g, seed, t, t.size, out)
    return out


def ref_get_hg_lut(lut, cosv, angle):
    return ref_volume().ref_vol_get_hg_lut(np.ascontiguousarray(lut, np.float32).ravel(), cosv, angle)


def ref_bake_voxels(data, R, max_density, alpha, light_dir, bake_res, seed, voxels):
    v = np.ascontiguousarray(voxels, np.int64)
    out = np.empty(v.size, np.float32)
    ref_volume().ref_vol_bake_voxels(np.ascontiguousarray(data, np.float32).ravel(), R, max_density, alpha,
                                     np.asarray(light_dir, np.float32), bake_res, seed, v, v.size, out)
    return out


def ref_load_hdr(path):
    """The reference's RGBE loader: float32 [ry, rx, 4], or None if it fails."""
    rx, ry = C.c_uint(), C.c_uint()
    if ref_volume().ref_vol_load_hdr(path.encode(), C.byref(rx), C.byref(ry), None, 0) != 0:
        return None
    out = np.empty((ry.value, rx.value, 4), np.float32)
    ref_volume().ref_vol_load_hdr(path.encode(), C.byref(rx), C.byref(ry), out.ctypes.data, out.size)
    return out


def env_light(scene, frame, seed, light_dir, light_color, n=0):
    """The light of predictor launch `frame` with the scene's environment
    map: the coin is the first uniform of Philox stream (6, 0, 0, frame,
    seed), as the library draws it.  Returns (L, C)."""
    L = np.array(light_dir, np.float32)
    Cc = np.array(light_color, np.float32)
    coin = lib().orc_stream_uniform(6, 0, 0, frame, seed, 0)
    lib().orc_env_light(C.byref(scene.c), coin, n, L, Cc)
    return L, Cc


def baked_tr_voxels(scene, alpha, light_dir, bake_res, seed, voxels, replicate=True):
    """The oracle's Fill_BakeTR at voxels (index (x * B + y) * B + z)."""
    v = np.ascontiguousarray(voxels, np.int64)
    out = np.empty(v.size, np.float32)
    lib().orc_baked_tr(C.byref(scene.c), alpha, np.asarray(light_dir, np.float32), bake_res, seed,
                       1 if replicate else 0, v, v.size, out)
    return out


# ---------------------------------------------------------------------------
# numpy-level helpers
# ---------------------------------------------------------------------------
def mip_sizes():
    return [256 >> m for m in range(9)]


def tr_sizes():
    return [128 >> i for i in range(8)]


def split_levels(flat, sizes):
    out, off = [], 0
    for r in sizes:
        out.append(flat[off:off + r ** 3].reshape(r, r, r))
        off += r ** 3
    return out


def fbm_volume(R, seed, base_freq, octaves=6, gain=0.5):
    out = np.empty(R ** 3, np.float32)
    lib().orc_fbm_volume(out, R, seed, base_freq, octaves, gain)
    return out


def build_pyramid(data, R):
    out = np.empty(sum(r ** 3 for r in mip_sizes()), np.float32)
    lib().orc_build_pyramid(np.ascontiguousarray(data, np.float32).ravel(), R, out)
    return out


def tr_mips(mips, alpha, light_dir, levels=range(8)):
    out = np.zeros(sum(r ** 3 for r in tr_sizes()), np.float32)
    offs = np.cumsum([0] + [r ** 3 for r in tr_sizes()])
    L = np.asarray(light_dir, np.float32)
    for lv in levels:
        part = np.empty(tr_sizes()[lv] ** 3, np.float32)
        lib().orc_tr_mip_level(mips, lv, alpha, L, part)
        out[offs[lv]:offs[lv + 1]] = part
    return out


def hg_lut_texels(g, seed, texels):
    t = np.ascontiguousarray(texels, np.int32)
    out = np.empty(t.size, np.float32)
    lib().orc_hg_lut_texels(g, seed, t, t.size, out)
    return out


def stencil_tables():
    off = np.empty(192, np.float32)
    layer = np.empty(192, np.int32)
    typ = np.empty(192, np.int32)
    li = np.empty(192, np.int32)
    v = np.empty(192, np.float32)
    lib().orc_stencil_tables(off, layer, typ, li, v)
    return off, layer, typ, li, v


def lut_rows_needed():
    """LUT texel indices read by the gather: the two rows around each stencil v."""
    _, _, _, _, v = stencil_tables()
    rows = set()
    for vv in v:
        y = int(np.floor(vv * 512 - 0.5))
        for r in (y, y + 1):
            rows.add(min(max(r, 0), 511))
    rows = sorted(rows)
    return rows, np.concatenate([np.arange(r * 512, (r + 1) * 512, dtype=np.int32) for r in rows])


class SceneBuf:
    """Host arrays for one scene plus the ctypes struct pointing at them."""

    def __init__(self, density, res, max_density, mips=None, tr=None, lut=None, baked=None, baked_res=0,
                 scatter_rate=(1.001, 1.001, 1.001), tr_scale=1.0, sky=(0.0, 0.0, 0.0), hdri=None, env_exp=1.0):
        """hdri: an equirect environment map, float32 [h, w, 4] (RGBA rows),
        or None for the constant sky."""
        keep = lambda a: None if a is None else np.ascontiguousarray(a, np.float32).ravel()
        self.density, self.mips, self.tr, self.lut, self.baked = map(keep, (density, mips, tr, lut, baked))
        self.res, self.max_density, self.baked_res = res, float(max_density), baked_res
        self.scatter_rate = np.asarray(scatter_rate, np.float32)
        self.tr_scale = float(tr_scale)
        self.sky = np.asarray(sky, np.float32)
        self.hdri = None if hdri is None else np.ascontiguousarray(hdri, np.float32)
        hh, hw = (0, 0) if hdri is None else self.hdri.shape[:2]
        self.env_exp = float(env_exp)
        ptr = lambda a: None if a is None else a.ctypes.data
        self.c = Scene(ptr(self.density), res, self.max_density, ptr(self.mips), ptr(self.tr), ptr(self.lut),
                       ptr(self.baked), baked_res, F3(*self.scatter_rate), self.tr_scale, F3(*self.sky),
                       ptr(self.hdri), hw, hh, self.env_exp)

    def bind_ref(self):
        ref().ref_bind_scene(self.c.density, self.res, self.max_density, self.c.mips, self.c.tr_mips,
                             self.c.hg_lut, self.c.baked_tr, self.baked_res, self.scatter_rate, self.tr_scale,
                             self.sky, self.c.hdri, self.c.hdri_w, self.c.hdri_h, self.env_exp)


def make_view(width, height, ori, up, right, light_dir, light_color=(1, 1, 1), alpha=64.0, g=0.857,
              multi_scatter=256, spp=32, seed=0, frame=0):
    return View(width, height, F3(*ori), F3(*up), F3(*right), F3(*light_dir), F3(*light_color), alpha, g,
                multi_scatter, spp, seed, frame)


def predict_pixels(scene, view, pixels, want_features=False):
    px = np.ascontiguousarray(pixels, np.int32)
    n = px.size
    rgba = np.empty((n, 4), np.float32)
    feat = np.empty((n, 576), np.float32) if want_features else None
    gam = np.empty(n, np.float32) if want_features else None
    hit = np.empty((n, 4), np.float32) if want_features else None
    p = lambda a: None if a is None else a.ctypes.data
    lib().orc_predict_pixels(C.byref(scene.c), C.byref(view), px, n, rgba, p(feat), p(gam), p(hit))
    return (rgba, feat, gam, hit) if want_features else rgba


def trace_pixels(scene, view, pixels):
    px = np.ascontiguousarray(pixels, np.int32)
    n = px.size
    rgba = np.empty((n, 4), np.float32)
    s = np.empty((n, 3), np.float64)
    s2 = np.empty((n, 3), np.float64)
    lib().orc_trace_pixels(C.byref(scene.c), C.byref(view), px, n, rgba, s.ctypes.data, s2.ctypes.data)
    return rgba, s, s2


def trace_rays(scene, view, ori, dir):
    """GetRadiances (PT) for explicit rays: FP64 sums of L and L^2 over view.spp."""
    ori = np.ascontiguousarray(ori, np.float32).reshape(-1, 3)
    dir = np.ascontiguousarray(dir, np.float32).reshape(-1, 3)
    n = ori.shape[0]
    s = np.empty((n, 3), np.float64)
    s2 = np.empty((n, 3), np.float64)
    lib().orc_trace_rays(C.byref(scene.c), C.byref(view), ori.ctypes.data, dir.ctypes.data, n, s.ctypes.data,
                         s2.ctypes.data)
    return s, s2


def get_samples(scene, alpha, ori, dir, ldir, g, scatter, light_color, multi_scatter, spp, seed):
    ori = np.ascontiguousarray(ori, np.float32).reshape(-1, 3)
    n = ori.shape[0]
    arr = lambda x, k: np.ascontiguousarray(np.broadcast_to(np.asarray(x, np.float32), (n, k) if k > 1 else (n,)))
    a, d, L, gg, sc = arr(alpha, 1), arr(dir, 3), arr(ldir, 3), arr(g, 1), arr(scatter, 1)
    out = np.empty((n, 3), np.float32)
    lib().orc_get_samples(C.byref(scene.c), a.ctypes.data, ori.ctypes.data, d.ctypes.data, L.ctypes.data,
                          gg.ctypes.data, sc.ctypes.data, n, F3(*light_color), multi_scatter, spp, seed,
                          out.ctypes.data)
    return out


def get_trs(scene, alpha, ori, dir, light_dir, light_color, g, spp, seed):
    ori = np.ascontiguousarray(ori, np.float32).reshape(-1, 3)
    dir = np.ascontiguousarray(dir, np.float32).reshape(-1, 3)
    n = ori.shape[0]
    out = np.empty((n, 3), np.float32)
    lib().orc_get_trs(C.byref(scene.c), alpha, ori.ctypes.data, dir.ctypes.data, n, F3(*light_dir),
                      F3(*light_color), g, spp, seed, out.ctypes.data)
    return out


def frame_pt(scene, view, fnum, checker, flip, target, histo):
    """Interactive PT frame on copies of (target [H, W, 3], histo [H, W, 33])."""
    t = np.ascontiguousarray(target, np.float32).copy()
    h = np.ascontiguousarray(histo, np.float32).copy()
    lib().orc_frame_pt(C.byref(scene.c), C.byref(view), fnum, checker, flip, t.ctypes.data, h.ctypes.data)
    return t, h


def frame_finish(target, histo, frame_num, flip, predict, denoise, exposure, tone):
    t = np.ascontiguousarray(target, np.float32)
    h = np.ascontiguousarray(histo, np.float32).copy()
    H, W = t.shape[:2]
    out = np.empty((H, W), np.uint32)
    lib().orc_frame_finish(t.ctypes.data, h.ctypes.data, W, H, frame_num, flip, predict, denoise, exposure, tone,
                           out.ctypes.data)
    return out, h


def gather_tiles(scene, view, px, py):
    """GatherData: [view.width * view.height, 773] tile features."""
    out = np.empty((view.width * view.height, 773), np.float32)
    lib().orc_gather_tiles(C.byref(scene.c), C.byref(view), px, py, out.ctypes.data)
    return out


def mlp_f32(feat, gamma, g, sr):
    feat = np.ascontiguousarray(feat, np.float32)
    n = feat.shape[0]
    out = np.empty((n, 3), np.float32)
    lib().orc_mlp_f32(feat, np.ascontiguousarray(gamma, np.float32), g, np.asarray(sr, np.float32), n, out)
    return out


def mlp_f64(feat, gamma, g, sr):
    feat = np.ascontiguousarray(feat, np.float32)
    n = feat.shape[0]
    out = np.empty((n, 3), np.float64)
    lib().orc_mlp_f64(feat, np.ascontiguousarray(gamma, np.float32), g, np.asarray(sr, np.float32), n, out)
    return out


def ref_mlp(feat, gamma, g, sr):
    feat = np.ascontiguousarray(feat, np.float32)
    n = feat.shape[0]
    out = np.empty((n, 3), np.float32)
    ref().ref_mlp(feat, np.ascontiguousarray(gamma, np.float32), g, np.asarray(sr, np.float32), n, out)
    return out
