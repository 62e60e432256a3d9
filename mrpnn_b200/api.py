"""Python mirror of the reference's render API over the C ABI (include/mrpnn.h).

The reference's public interface is the C++ pair ``VolumeRender``
(core/volume.hpp:45-155) and ``Camera`` (core/camera.hpp:29-43); this module
keeps their method names, argument meaning and defaults, so a script written
against them reads the same.  All work runs in ``libmrpnn_b200.so`` on the
GPU; importing works without a GPU, but any call that needs the device raises
``MrpError`` when no sm_100 device is present -- there is no CPU path.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmrpnn_b200.so")
MODEL_PATH = os.path.join(HERE, "data", "mrpnn_model.bin")

# mrp_status
OK, ERR_INVALID, ERR_NO_DEVICE, ERR_CUDA, ERR_OOM, ERR_NOT_READY, ERR_UNSUPPORTED, ERR_IO, ERR_BUDGET, ERR_TIMEOUT = range(10)
STATUS_NAMES = ["OK", "INVALID", "NO_DEVICE", "CUDA", "OOM", "NOT_READY", "UNSUPPORTED", "IO", "BUDGET", "TIMEOUT"]
FP32, BF16, FP8 = 0, 1, 2
RES_DENSITY, RES_MIP, RES_TR, RES_LUT, RES_BAKED_TR, RES_OCCUPANCY = range(6)

F3 = C.c_float * 3


class MrpError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"mrp {STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else status}: {msg}")
        self.status = status


class Params(C.Structure):
    _fields_ = [("scatter_rate", F3), ("tr_scale", C.c_float), ("sky", F3), ("env_exp", C.c_float),
                ("bake_res", C.c_int), ("bake_replicate_seeding", C.c_int), ("precision", C.c_int),
                ("seed", C.c_uint32), ("nee_mode", C.c_int), ("tracer_filter", C.c_int),
                ("gather_filter", C.c_int)]


class View(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("ori", F3), ("up", F3), ("right", F3),
                ("light_dir", F3), ("light_color", F3), ("alpha", C.c_float), ("g", C.c_float),
                ("multi_scatter", C.c_int), ("spp", C.c_int), ("seed", C.c_uint32), ("frame_offset", C.c_int)]


class VolumeInfo(C.Structure):
    _fields_ = [("res", C.c_int), ("max_density", C.c_float), ("has_pyramid", C.c_int), ("has_lut", C.c_int),
                ("has_tr", C.c_int), ("has_baked_tr", C.c_int), ("lut_g", C.c_float), ("tr_alpha", C.c_float),
                ("tr_light", F3), ("device_bytes", C.c_size_t)]


class ServeConfig(C.Structure):
    _fields_ = [("memory_budget", C.c_size_t), ("max_slots", C.c_int), ("precision", C.c_int),
                ("slot_pixels", C.c_size_t)]


class Request(C.Structure):
    _fields_ = [("volume", C.c_void_p), ("view", View), ("out_rgba", C.c_void_p), ("out_is_device", C.c_int)]


class RequestTiming(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("submit_ms", "admit_ms", "features_ms", "network_ms", "done_ms")]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_ulonglong), ("completed", C.c_ulonglong), ("failed", C.c_ulonglong),
                ("batches", C.c_ulonglong), ("batched_requests", C.c_ulonglong), ("max_batch", C.c_int),
                ("bytes_in_use", C.c_size_t), ("peak_bytes", C.c_size_t)]


FILL_FN = C.CFUNCTYPE(C.c_float, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_void_p)

# Every symbol include/mrpnn.h declares, with its ctypes signature.
_SIGS = {
    "mrp_init": ([C.c_int, C.c_char_p], C.c_int),
    "mrp_last_error": ([], C.c_char_p),
    "mrp_version": ([], C.c_char_p),
    "mrp_debug_alloc_calls": ([], C.c_ulonglong),
    "mrp_load_model": ([C.c_char_p], C.c_int),
    "mrp_default_params": ([C.POINTER(Params)], None),
    "mrp_volume_create": ([C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "mrp_volume_create_ex": ([C.c_int, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "mrp_render_start": ([C.c_void_p, C.POINTER(View), C.c_int, C.c_int, C.c_void_p, C.c_int], C.c_int),
    "mrp_render_wait": ([C.c_void_p, C.c_int], C.c_int),
    "mrp_volume_destroy": ([C.c_void_p], C.c_int),
    "mrp_volume_set_data": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int], C.c_int),
    "mrp_volume_fill": ([C.c_void_p, FILL_FN, C.c_void_p], C.c_int),
    "mrp_volume_generate_fbm": ([C.c_void_p, C.c_uint32, C.c_float, C.c_int, C.c_float], C.c_int),
    "mrp_volume_update": ([C.c_void_p, C.c_int], C.c_int),
    "mrp_volume_set_max_density": ([C.c_void_p, C.c_float], C.c_int),
    "mrp_volume_get_info": ([C.c_void_p, C.POINTER(VolumeInfo)], C.c_int),
    "mrp_set_params": ([C.c_void_p, C.POINTER(Params)], C.c_int),
    "mrp_get_params": ([C.c_void_p, C.POINTER(Params)], C.c_int),
    "mrp_volume_read": ([C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_size_t), C.c_int], C.c_int),
    "mrp_update_hg_lut": ([C.c_void_p, C.c_float], C.c_int),
    "mrp_update_tr": ([C.c_void_p, F3, C.c_float], C.c_int),
    "mrp_update_baked_tr": ([C.c_void_p, F3, C.c_float], C.c_int),
    "mrp_render": ([C.c_void_p, C.POINTER(View), C.c_int, C.c_int, C.c_void_p, C.c_int], C.c_int),
    "mrp_last_render_ms": ([C.c_void_p, C.POINTER(C.c_float)], C.c_int),
    "mrp_last_render_stages": ([C.c_void_p, C.POINTER(C.c_float)], C.c_int),
    "mrp_render_counters": ([C.c_void_p, C.POINTER(View), C.c_int, C.POINTER(C.c_ulonglong)], C.c_int),
    "mrp_predict_features": ([C.c_void_p, C.c_void_p, C.c_float, F3, C.c_int, C.c_void_p, C.c_int, C.c_int], C.c_int),
    "mrp_predict_features_noalloc": ([C.c_void_p, C.c_void_p, C.c_float, F3, C.c_int, C.c_void_p, C.c_int], C.c_int),
    "mrp_gather_features": ([C.c_void_p, C.c_void_p, C.c_void_p, F3, C.c_float, C.c_float, C.c_int, C.c_void_p,
                             C.c_void_p, C.c_int], C.c_int),
    "mrp_first_hit": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_void_p, C.c_int], C.c_int),
    "mrp_tc_gemm_check": ([C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "mrp_measure_l1_rate": ([C.POINTER(C.c_float)], C.c_int),
    "mrp_measure_l2_rate": ([C.POINTER(C.c_float)], C.c_int),
    "mrp_render_predict_debug": ([C.c_void_p, C.POINTER(View), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "mrp_hdri_file_read": ([C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p, C.c_size_t], C.c_int),
    "mrp_volume_set_hdri": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int], C.c_int),
    "mrp_volume_load_hdri": ([C.c_void_p, C.c_char_p], C.c_int),
    "mrp_hg_lut_lookup": ([C.c_void_p, C.c_float, C.c_float, C.POINTER(C.c_float)], C.c_int),
    "mrp_volume_file_read": ([C.c_char_p, C.POINTER(C.c_int), C.c_void_p, C.c_size_t], C.c_int),
    "mrp_volume_file_write_bin": ([C.c_char_p, C.c_void_p, C.c_int], C.c_int),
    "mrp_volume_load": ([C.c_char_p, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "mrp_render_views": ([C.c_void_p, C.POINTER(View), C.c_int, C.POINTER(C.c_void_p), C.c_int], C.c_int),
    "mrp_get_radiances": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, F3, F3, C.c_float, C.c_int, C.c_float,
                           C.c_int, C.c_int, C.c_void_p, C.c_int], C.c_int),
    "mrp_get_samples": ([C.c_void_p] + [C.c_void_p] * 6 + [C.c_int, F3, C.c_int, C.c_int, C.c_uint32, C.c_void_p,
                                                            C.c_int], C.c_int),
    "mrp_get_trs": ([C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_int, F3, F3, C.c_float, C.c_int, C.c_uint32,
                     C.c_void_p, C.c_int], C.c_int),
    "mrp_render_interactive": ([C.c_void_p, C.POINTER(View), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "mrp_gather_tiles": ([C.c_void_p, C.POINTER(View), C.c_int, C.c_int, C.c_void_p, C.c_int], C.c_int),
    "mrp_serve_default_config": ([C.POINTER(ServeConfig)], None),
    "mrp_serve_open": ([C.POINTER(ServeConfig), C.POINTER(C.c_void_p)], C.c_int),
    "mrp_serve_submit": ([C.c_void_p, C.POINTER(Request), C.POINTER(C.c_uint64)], C.c_int),
    "mrp_serve_poll": ([C.c_void_p, C.c_uint64, C.c_int, C.POINTER(C.c_int), C.POINTER(RequestTiming)], C.c_int),
    "mrp_serve_stats_get": ([C.c_void_p, C.POINTER(ServeStats)], C.c_int),
    "mrp_serve_close": ([C.c_void_p], C.c_int),
}

_lib = None
_initialized = False


def lib():
    """Loads libmrpnn_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MrpError(ERR_NOT_READY, f"{LIB_PATH} is missing: build it with `python -m mrpnn_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(status):
    if status != OK:
        raise MrpError(status, lib().mrp_last_error().decode(errors="replace"))


def init(device=0, model_path=None):
    """mrp_init: selects the CUDA device and loads the network weights."""
    global _initialized
    _check(lib().mrp_init(device, model_path.encode() if model_path else MODEL_PATH.encode()))
    _initialized = True


def _ensure_init():
    if not _initialized:
        init()


def _f3(v):
    v = [float(x) for x in v]
    return F3(*v)


def _ptr(a):
    """(pointer, is_device) of a numpy array or a CUDA torch tensor."""
    if isinstance(a, np.ndarray):
        return a.ctypes.data, 0
    if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
        return a.data_ptr(), 1
    raise TypeError("expected a numpy array or a CUDA tensor")


def _host_f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        a = a.reshape(shape)
    return a


FEATURES_PER_SET = 576   # X_Val, X_Val_Sub, X_Val_Hg: 3 x 192 stencil points


def _feature_sets(feat, gamma):
    """Host feature sets as contiguous float32 ([n, 576], [n], n), or
    ValueError when the shapes disagree: the C ABI reads n * 576 and n floats
    from these pointers, so a malformed array must never reach it."""
    feat = np.ascontiguousarray(feat, dtype=np.float32)
    gamma = np.ascontiguousarray(gamma, dtype=np.float32)
    if feat.ndim != 2 or feat.shape[1] != FEATURES_PER_SET:
        raise ValueError(f"feat must be [n, {FEATURES_PER_SET}]; got {feat.shape}")
    if gamma.ndim != 1 or gamma.shape[0] != feat.shape[0]:
        raise ValueError(f"gamma must be [n] with n = {feat.shape[0]}; got {gamma.shape}")
    return feat, gamma, feat.shape[0]


def default_params():
    p = Params()
    lib().mrp_default_params(C.byref(p))
    return p


def predict_features(feat, gamma, g, scatter_rate, precision=FP32, out=None):
    """RadiancePredictInternal on n feature sets (feat [n, 576] = X_Val, X_Val_Sub,
    X_Val_Hg; gamma [n]) -> [n, 3].  Accepts numpy arrays (host) or CUDA tensors."""
    if isinstance(feat, np.ndarray):
        feat, gamma, n = _feature_sets(feat, gamma)
        if out is None:
            out = np.empty((n, 3), np.float32)
        elif not (isinstance(out, np.ndarray) and out.dtype == np.float32 and out.shape == (n, 3)
                  and out.flags.c_contiguous):
            raise ValueError(f"out must be a C-contiguous float32 array of shape ({n}, 3)")
        _ensure_init()
        _check(lib().mrp_predict_features(feat.ctypes.data, gamma.ctypes.data, float(g), _f3(scatter_rate), n,
                                          out.ctypes.data, int(precision), 0))
        return out
    import torch
    if not (isinstance(feat, torch.Tensor) and isinstance(gamma, torch.Tensor) and feat.is_cuda and gamma.is_cuda):
        raise TypeError("feat and gamma must both be numpy arrays or both CUDA tensors")
    if feat.dtype != torch.float32 or gamma.dtype != torch.float32 or not feat.is_contiguous() \
            or not gamma.is_contiguous():
        raise ValueError("feat and gamma must be contiguous float32 tensors")
    if feat.dim() != 2 or feat.shape[1] != FEATURES_PER_SET or gamma.numel() != feat.shape[0]:
        raise ValueError(f"feat must be [n, {FEATURES_PER_SET}] and gamma [n]; got {tuple(feat.shape)} "
                         f"and {tuple(gamma.shape)}")
    n = feat.shape[0]
    if out is None:
        out = torch.empty((n, 3), dtype=torch.float32, device=feat.device)
    elif not (isinstance(out, torch.Tensor) and out.is_cuda and out.dtype == torch.float32
              and tuple(out.shape) == (n, 3) and out.is_contiguous()):
        raise ValueError(f"out must be a contiguous float32 CUDA tensor of shape ({n}, 3)")
    _ensure_init()
    _check(lib().mrp_predict_features(feat.data_ptr(), gamma.data_ptr(), float(g), _f3(scatter_rate), n,
                                      out.data_ptr(), int(precision), 1))
    return out


def read_hdri(path):
    """mrp_hdri_file_read: a Radiance .hdr file as float32 [height, width, 4]
    (RGBA rows top to bottom, alpha 0), as the reference's loader reads it."""
    w, h = C.c_int(), C.c_int()
    _check(lib().mrp_hdri_file_read(path.encode(), C.byref(w), C.byref(h), None, 0))
    out = np.empty((h.value, w.value, 4), np.float32)
    _check(lib().mrp_hdri_file_read(path.encode(), C.byref(w), C.byref(h), out.ctypes.data, out.size))
    return out


def hg_lut_lookup(lut, cos_theta, angle):
    """mrp_hg_lut_lookup: VolumeRender::GetHGLut's read of a 512 x 512 HG
    table (host only)."""
    lut = _host_f32(lut).ravel()
    if lut.size != 512 * 512:
        raise ValueError("the HG table has 512 x 512 entries")
    out = C.c_float()
    _check(lib().mrp_hg_lut_lookup(lut.ctypes.data, float(cos_theta), float(angle), C.byref(out)))
    return out.value


def read_volume_file(path):
    """mrp_volume_file_read: a .bin / .txt / .vox volume as float32 [R, R, R]
    (z fastest), on the host; no device needed."""
    r = C.c_int()
    _check(lib().mrp_volume_file_read(path.encode(), C.byref(r), None, 0))
    out = np.empty((r.value,) * 3, np.float32)
    _check(lib().mrp_volume_file_read(path.encode(), C.byref(r), out.ctypes.data, out.size))
    return out


def write_volume_bin(path, data):
    """mrp_volume_file_write_bin: the reference's .bin cache format."""
    data = _host_f32(data)
    R = data.shape[0]
    assert data.shape == (R, R, R)
    _check(lib().mrp_volume_file_write_bin(path.encode(), data.ctypes.data, R))


def debug_alloc_calls():
    """mrp_debug_alloc_calls: CUDA allocation and free calls the library has
    made so far (device, stream-ordered and pinned host)."""
    return int(lib().mrp_debug_alloc_calls())


NOALLOC_MAX_POINTS = 2048   # MRP_NOALLOC_MAX_POINTS in include/mrpnn.h


def predict_features_noalloc(feat, gamma, g, scatter_rate, precision=FP32):
    """predict_features for host arrays through mrp_predict_features_noalloc,
    for callers that must not allocate device memory mid-render: the device
    copies, the output and the tensor-core network's counters sit in the
    library's fixed device array.  At most NOALLOC_MAX_POINTS feature sets
    per call."""
    feat, gamma, n = _feature_sets(feat, gamma)
    _ensure_init()
    out = np.empty((n, 3), np.float32)
    _check(lib().mrp_predict_features_noalloc(feat.ctypes.data, gamma.ctypes.data, float(g), _f3(scatter_rate), n,
                                              out.ctypes.data, int(precision)))
    return out


def measure_l1_rate():
    """mrp_measure_l1_rate: GB/s of cached 8-byte loads on this GPU."""
    _ensure_init()
    r = C.c_float()
    _check(lib().mrp_measure_l1_rate(C.byref(r)))
    return r.value


def measure_l2_rate():
    """mrp_measure_l2_rate: GB/s of 16-byte L2 reads (L1 bypassed) on this GPU."""
    _ensure_init()
    r = C.c_float()
    _check(lib().mrp_measure_l2_rate(C.byref(r)))
    return float(r.value)


def tc_gemm_check(A, B, fp8=False):
    """D = A B^T through one tcgen05.mma chain (A [128, k], B [n, k])."""
    _ensure_init()
    A = _host_f32(A)
    B = _host_f32(B)
    n, k = B.shape
    D = np.empty((128, n), np.float32)
    _check(lib().mrp_tc_gemm_check(1 if fp8 else 0, A.ctypes.data, B.ctypes.data, n, k, D.ctypes.data))
    return D


# density grid storage (mrp_storage)
STORAGE = {"fp32": 0, "fp16": 1}


class VolumeRender:
    """VolumeRender (core/volume.hpp:45-155) over a device-resident volume handle."""
    PT, RPNN, MRPNN = 0, 1, 2

    def __init__(self, resolution, cacheTR=False, write_cache=True, storage="fp32"):
        """VolumeRender(int resolution) or VolumeRender(string path, bool
        cacheTR) (core/volume.cu:948-967): a path loads a .bin / .txt / .vox
        file (LoadData) and runs Update; cacheTR has no effect here (the baked
        TR grid is sized by SetBakeResolution, not by the load).  storage
        "fp16" keeps a new grid in half precision (values rounded to nearest
        on the way in; renders as an fp32 grid of the rounded values)."""
        if storage not in STORAGE:
            raise ValueError(f"storage must be one of {sorted(STORAGE)}")
        _ensure_init()
        h = C.c_void_p()
        if isinstance(resolution, (str, bytes, os.PathLike)):
            _check(lib().mrp_volume_load(os.fsencode(resolution), 1 if write_cache else 0, C.byref(h)))
            self._h = h
            self.resolution = int(self.info().res)
        else:
            _check(lib().mrp_volume_create_ex(int(resolution), STORAGE[storage], C.byref(h)))
            self._h = h
            self.resolution = int(resolution)
        self._params = default_params()
        self._view_seed = 0
        self._inflight = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.mrp_volume_destroy(h)
            self._h = None

    def close(self):
        self.__del__()

    # -- data -------------------------------------------------------------
    def set_data(self, data):
        """Full grid, index (x*R + y)*R + z (SetData storage, core/volume.cu:1178)."""
        if isinstance(data, np.ndarray):
            data = _host_f32(data).ravel()
            if data.size != self.resolution ** 3:
                raise ValueError("data size does not match the resolution")
            _check(lib().mrp_volume_set_data(self._h, data.ctypes.data, self.resolution, 0))
        else:
            _check(lib().mrp_volume_set_data(self._h, data.data_ptr(), self.resolution, 1))

    def SetDatas(self, func):
        """SetDatas(FillFunc) (core/volume.cu:1182): func(x, y, z, u, v, w) -> float.
        func may take numpy index/coordinate grids (vectorised) or scalars."""
        R = self.resolution
        i = np.arange(R)
        x, y, z = np.meshgrid(i, i, i, indexing="ij")
        u = ((x + 0.5) / R).astype(np.float32)
        v = ((y + 0.5) / R).astype(np.float32)
        w = ((z + 0.5) / R).astype(np.float32)
        try:
            vals = np.asarray(func(x, y, z, u, v, w), dtype=np.float32)
            if vals.shape != x.shape:
                raise ValueError
        except Exception:
            cb = FILL_FN(lambda a, b, c, uu, vv, ww, _u: float(func(a, b, c, uu, vv, ww)))
            _check(lib().mrp_volume_fill(self._h, cb, None))
            return
        self.set_data(vals)

    def generate_fbm(self, seed, base_freq, octaves=6, gain=0.5):
        """Synthetic fBm cloud on the device (benchmark volumes)."""
        _check(lib().mrp_volume_generate_fbm(self._h, int(seed), float(base_freq), int(octaves), float(gain)))

    def Update(self, process_mips=True, need_reset_datas_dev=True):
        _check(lib().mrp_volume_update(self._h, 1 if process_mips else 0))

    @property
    def max_density(self):
        return self.info().max_density

    @max_density.setter
    def max_density(self, value):
        _check(lib().mrp_volume_set_max_density(self._h, float(value)))

    def info(self):
        inf = VolumeInfo()
        _check(lib().mrp_volume_get_info(self._h, C.byref(inf)))
        return inf

    def read(self, which, level=0):
        n = C.c_size_t()
        _check(lib().mrp_volume_read(self._h, which, level, None, C.byref(n), 0))
        out = np.empty(n.value, np.uint8 if which == RES_OCCUPANCY else np.float32)
        _check(lib().mrp_volume_read(self._h, which, level, out.ctypes.data, None, 0))
        return out

    # -- settings (core/volume.cu:1732-1765) ----------------------------------
    def _push(self):
        _check(lib().mrp_set_params(self._h, C.byref(self._params)))

    def SetScatterRate(self, rate):
        r = [rate] * 3 if np.isscalar(rate) else list(rate)
        self._params.scatter_rate = _f3(r)
        self._push()

    def SetTrScale(self, scale):
        self._params.tr_scale = float(scale)
        self._push()

    def SetEnvExp(self, exp):
        self._params.env_exp = float(exp)
        self._push()

    def SetSky(self, radiance):
        r = [radiance] * 3 if np.isscalar(radiance) else list(radiance)
        self._params.sky = _f3(r)
        self._push()

    def SetPrecision(self, precision):
        self._params.precision = int(precision)
        self._push()

    def GetPrecision(self):
        return int(self._params.precision)

    def SetBakeResolution(self, res, replicate_reference_seeding=True):
        self._params.bake_res = int(res)
        self._params.bake_replicate_seeding = 1 if replicate_reference_seeding else 0
        self._push()

    def SetSeed(self, seed):
        self._params.seed = int(seed)
        self._push()

    def SetTracerFilter(self, hardware):
        """The frame tracer's free-flight density fetch: False (default)
        software trilinear in the reference's float order; True the texture
        unit's trilinear filter, as the reference's own tex3D."""
        self._params.tracer_filter = 1 if hardware else 0
        self._push()

    def SetGatherFilter(self, hardware):
        """The stencil gather of the BF16 / FP8 forms: True (default) the
        texture unit's trilinear / bilinear filters on the mip and TR levels
        (and the LUT for the light ray's points), as the reference's own
        tex3D / tex2D sampling; False software filters with fp32 weights.  The
        FP32 form always filters in software."""
        self._params.gather_filter = 1 if hardware else 0
        self._push()

    def SetNeeMode(self, unbiased):
        """PT next-event estimation: False (default) samples the baked TR grid
        like the reference; True takes one ratio-tracking Tr() estimate per
        vertex (unbiased; no bake)."""
        self._params.nee_mode = 1 if unbiased else 0
        self._push()

    # -- caches -------------------------------------------------------------------
    def UpdateHGLut(self, g):
        _check(lib().mrp_update_hg_lut(self._h, float(g)))

    def SetHDRI(self, path_or_map):
        """VolumeRender::SetHDRI (core/volume.cu:1696-1728): a .hdr file path,
        or an equirect map float32 [h, w, 4]; None clears it."""
        if path_or_map is None:
            _check(lib().mrp_volume_set_hdri(self._h, None, 0, 0))
        elif isinstance(path_or_map, str):
            _check(lib().mrp_volume_load_hdri(self._h, path_or_map.encode()))
        else:
            m = _host_f32(path_or_map)
            if m.ndim != 3 or m.shape[2] != 4:
                raise ValueError("the environment map is float32 [height, width, 4]")
            _check(lib().mrp_volume_set_hdri(self._h, m.ctypes.data, m.shape[1], m.shape[0]))

    def GetHGLut(self, cos, angle):
        """VolumeRender::GetHGLut (core/volume.cu:1424-1442) on the volume's
        current HG table (read back from the device once per table)."""
        key = float(self.info().lut_g)
        if getattr(self, "_lut_host_g", None) != key:
            self._lut_host = self.read(RES_LUT)[:512 * 512].copy()
            self._lut_host_g = key
        return hg_lut_lookup(self._lut_host, cos, angle)

    def Update_TR(self, lightDir, alpha=64.0, CPU=False):
        _check(lib().mrp_update_tr(self._h, _f3(lightDir), float(alpha)))

    def Update_CachedTR(self, lightDir, alpha):
        _check(lib().mrp_update_baked_tr(self._h, _f3(lightDir), float(alpha)))

    # -- rendering ----------------------------------------------------------------
    def make_view(self, size, ori, up, right, lightDir, g=0.857, alpha=1.0, lightColor=(1, 1, 1), multiScatter=512,
                  spp=32, seed=0, frame_offset=0):
        w, h = (size, size) if np.isscalar(size) else size
        return View(int(w), int(h), _f3(ori), _f3(up), _f3(right), _f3(lightDir), _f3(lightColor), float(alpha),
                    float(g), int(multiScatter), int(spp), int(seed), int(frame_offset))

    def Render(self, size, ori, up, right, lightDir, rt=PT, g=0.857, alpha=1.0, lightColor=(1, 1, 1),
               multiScatter=512, sampleNum=1024, spp=32, seed=0, out=None):
        """VolumeRender::Render (core/volume.cu:487-548) -> float32 [H, W, 4]
        (or into `out`, a numpy array or CUDA tensor of H*W*4 floats)."""
        view = self.make_view(size, ori, up, right, lightDir, g, alpha, lightColor, multiScatter, spp, seed)
        if out is None:
            out = np.empty((view.height, view.width, 4), np.float32)
        p, dev = _ptr(out)
        _check(lib().mrp_render(self._h, C.byref(view), int(rt), int(sampleNum), p, dev))
        return out

    def render_view(self, view, rt, sample_num, out):
        p, dev = _ptr(out)
        _check(lib().mrp_render(self._h, C.byref(view), int(rt), int(sample_num), p, dev))
        return out

    def render_view_start(self, view, rt, sample_num, out):
        """mrp_render_start: queues the render; `out` (pinned numpy or CUDA
        tensor) holds the result after render_wait()."""
        p, dev = _ptr(out)
        self._inflight.append(out)   # kept alive until the copy into it is done
        _check(lib().mrp_render_start(self._h, C.byref(view), int(rt), int(sample_num), p, dev))
        return out

    def render_wait(self, keep=0):
        """mrp_render_wait: every started render done (keep=0), or every one
        but the newest (keep=1)."""
        try:
            _check(lib().mrp_render_wait(self._h, int(keep)))
        finally:
            del self._inflight[:len(self._inflight) - keep if keep else None]

    # -- batch ray APIs (core/volume.cu:405-479, 710-834) ---------------------
    def GetRadiances(self, ori, dir, lightDir, lightColor=(1, 1, 1), alpha=1.0, multiScatter=1, g=0.0, sampleNum=1,
                     rt=None):
        """GetRadiances: radiance of explicit rays (PT or MRPNN), [n, 3]."""
        rt = self.PT if rt is None else rt
        ori = _host_f32(ori).reshape(-1, 3)
        dir = _host_f32(dir).reshape(-1, 3)
        out = np.empty((ori.shape[0], 3), np.float32)
        _check(lib().mrp_get_radiances(self._h, ori.ctypes.data, dir.ctypes.data, ori.shape[0], _f3(lightDir),
                                       _f3(lightColor), float(alpha), int(multiScatter), float(g), int(sampleNum),
                                       int(rt), out.ctypes.data, 0))
        return out

    def GetSamples(self, alpha, ori, dir, lightDir, g, scatter, lightColor=(1, 1, 1), multiScatter=1, sampleNum=1,
                   seed=0):
        """GetSamples: the training-data generator, per-task arrays, [n, 3]."""
        ori = _host_f32(ori).reshape(-1, 3)
        n = ori.shape[0]
        dir = _host_f32(dir).reshape(n, 3)
        L = _host_f32(lightDir).reshape(n, 3)
        a = _host_f32(np.broadcast_to(np.asarray(alpha, np.float32), (n,)))
        gg = _host_f32(np.broadcast_to(np.asarray(g, np.float32), (n,)))
        sc = _host_f32(np.broadcast_to(np.asarray(scatter, np.float32), (n,)))
        out = np.empty((n, 3), np.float32)
        _check(lib().mrp_get_samples(self._h, a.ctypes.data, ori.ctypes.data, dir.ctypes.data, L.ctypes.data,
                                     gg.ctypes.data, sc.ctypes.data, n, _f3(lightColor), int(multiScatter),
                                     int(sampleNum), int(seed), out.ctypes.data, 0))
        return out

    def GetTrs(self, alpha, ori, dir, lightDir, lightColor=(1, 1, 1), g=0.0, sampleNum=1, seed=0):
        """GetTrs: light colour x pi x mean Tr() x HG toward the light, [n, 3]."""
        ori = _host_f32(ori).reshape(-1, 3)
        dir = _host_f32(dir).reshape(-1, 3)
        out = np.empty((ori.shape[0], 3), np.float32)
        _check(lib().mrp_get_trs(self._h, float(alpha), ori.ctypes.data, dir.ctypes.data, ori.shape[0],
                                 _f3(lightDir), _f3(lightColor), float(g), int(sampleNum), int(seed),
                                 out.ctypes.data, 0))
        return out

    def GatherData(self, size, ori, up, right, lightDir, alpha=1.0, g=0.0, pixelOffset=(0, 0), seed=0, frame=0):
        """GatherData (core/volume.cu:630-700): [tiles_y * tiles_x, 773] tile
        features for a size = (tiles_x, tiles_y) grid of 8 x 8-pixel tiles."""
        view = self.make_view(size, ori, up, right, lightDir, g, alpha, seed=seed, frame_offset=frame)
        out = np.empty((view.width * view.height, 773), np.float32)
        _check(lib().mrp_gather_tiles(self._h, C.byref(view), int(pixelOffset[0]), int(pixelOffset[1]),
                                      out.ctypes.data, 0))
        return out

    def render_views(self, views, outs=None):
        """mrp_render_views: MRPNN images of several views (sharing light,
        alpha and g) with one batched network launch; numpy outputs by
        default, or a list of CUDA tensors."""
        n = len(views)
        arr = (View * n)(*views)
        if outs is None:
            outs = [np.empty((w.height, w.width, 4), np.float32) for w in views]
        ptrs, devs = zip(*[_ptr(o) for o in outs])
        if len(set(devs)) != 1:
            raise ValueError("outputs must be all host or all device buffers")
        parr = (C.c_void_p * n)(*ptrs)
        _check(lib().mrp_render_views(self._h, arr, n, parr, devs[0]))
        return outs

    def last_render_ms(self):
        ms = C.c_float()
        _check(lib().mrp_last_render_ms(self._h, C.byref(ms)))
        return ms.value

    def render_counters(self, view, rt):
        c = (C.c_ulonglong * 4)()
        _check(lib().mrp_render_counters(self._h, C.byref(view), int(rt), c))
        return [int(x) for x in c]

    def last_render_stages(self):
        ms = (C.c_float * 3)()
        _check(lib().mrp_last_render_stages(self._h, ms))
        return list(ms)

    # -- parity pieces ------------------------------------------------------------
    def gather_features(self, pos, bases, light_dir, g, alpha):
        pos = _host_f32(pos).reshape(-1, 3)
        bases = _host_f32(bases).reshape(-1, 12)
        n = pos.shape[0]
        feat = np.empty((n, 576), np.float32)
        gam = np.empty(n, np.float32)
        _check(lib().mrp_gather_features(self._h, pos.ctypes.data, bases.ctypes.data, _f3(light_dir), float(g),
                                         float(alpha), n, feat.ctypes.data, gam.ctypes.data, 0))
        return feat, gam

    def predict_debug(self, view):
        """One MRPNN launch at the volume's precision with its intermediates:
        (rgba [n,4], aux [n,20], feat [n,576]); BF16 / FP8 return the fp16
        features their tensor-core network reads, widened to float."""
        n = view.width * view.height
        rgba = np.empty((n, 4), np.float32)
        aux = np.empty((n, 20), np.float32)
        feat = np.empty((n, 576), np.float32)
        _check(lib().mrp_render_predict_debug(self._h, C.byref(view), rgba.ctypes.data, aux.ctypes.data,
                                              feat.ctypes.data, 0))
        return rgba, aux, feat

    def first_hit(self, ori, dirs, alpha):
        ori = _host_f32(ori).reshape(-1, 3)
        dirs = _host_f32(dirs).reshape(-1, 3)
        n = dirs.shape[0]
        if ori.shape[0] == 1 and n > 1:
            ori = np.ascontiguousarray(np.repeat(ori, n, axis=0))
        out = np.empty((n, 4), np.float32)
        _check(lib().mrp_first_hit(self._h, ori.ctypes.data, dirs.ctypes.data, float(alpha), n, out.ctypes.data, 0))
        return out


def camera_frame(position):
    """Camera::SetPosition (core/camera.cu:176-192): look-at-origin frame."""
    ori = np.asarray(position, np.float32)
    fwd = -ori / np.float32(np.sqrt(np.float32(np.dot(ori, ori))))
    right = np.cross(np.array([0, 1, 0], np.float32), fwd).astype(np.float32)
    right = right / np.float32(np.sqrt(np.float32(np.dot(right, right))))
    up = np.cross(fwd, right).astype(np.float32)
    if position[0] == 0 and position[2] == 0:
        right = np.array([1, 0, 0], np.float32)
        up = np.array([0, 0, 1 if position[1] > 0 else -1], np.float32)
    return ori, up, right


class Camera:
    """Camera (core/camera.hpp:29-43).  fov_deg scales right/up by tan(fov/2)
    (the reference's unit vectors give 90 degrees)."""

    def __init__(self, volume, name="test camera", position=(0.75, 0.75, 0.75), resolution=512, fov_deg=90.0):
        self.volume = volume
        self.name = name
        self.resolution = resolution
        self.fov_deg = fov_deg
        self.SetPosition(position)

    def SetPosition(self, position):
        self.ori, self.up, self.right = camera_frame(position)

    def GetPosition(self):
        return self.ori

    def SetVolume(self, volume):
        self.volume = volume

    def _scaled(self):
        s = np.float32(np.tan(np.deg2rad(self.fov_deg) / 2))
        return (self.up * s).astype(np.float32), (self.right * s).astype(np.float32)

    def Render(self, lightDir, lightColor=(1, 1, 1), alpha=1.0, multiScatter=1, g=0.0, sampleNum=1,
               rt=VolumeRender.PT, **kw):
        up, right = self._scaled()
        return self.volume.Render((self.resolution, self.resolution), self.ori, up, right, lightDir, rt, g, alpha,
                                  lightColor, multiScatter, sampleNum, **kw)

    def RenderToFile(self, path, lightDir, lightColor=(1, 1, 1), alpha=1.0, multiScatter=1, g=0.0, sampleNum=1,
                     tone=None, rt=VolumeRender.PT, exp=1.0, **kw):
        """Camera::RenderToFile (core/camera.cu:229-257): saturate to 8 bit and
        write `path`.png; like the reference it ignores `tone` and `exp`."""
        img = self.Render(lightDir, lightColor, alpha, multiScatter, g, sampleNum, rt, **kw)
        rgb = (np.clip(img[..., :3], 0.0, 1.0) * 255).astype(np.uint8)
        rgba = np.concatenate([rgb, np.full(rgb.shape[:2] + (1,), 255, np.uint8)], axis=-1)
        from PIL import Image
        Image.fromarray(rgba, "RGBA").save(path + ".png")
        return img


class Server:
    """The serving loop (mrp_serve_*): MRPNN requests on resident volumes with
    memory-budget admission and batched network launches.  Output buffers are
    numpy arrays (pinned or pageable) or CUDA tensors; they must stay alive
    until the ticket is polled done, which this wrapper takes care of."""

    def __init__(self, memory_budget=None, max_slots=16, precision=BF16, slot_pixels=0):
        _ensure_init()
        cfg = ServeConfig()
        lib().mrp_serve_default_config(C.byref(cfg))
        if memory_budget is not None:
            cfg.memory_budget = int(memory_budget)
        cfg.max_slots = int(max_slots)
        cfg.precision = int(precision)
        cfg.slot_pixels = int(slot_pixels)
        h = C.c_void_p()
        _check(lib().mrp_serve_open(C.byref(cfg), C.byref(h)))
        self._h = h
        self._outs = {}

    def submit(self, volume, view, out=None):
        """Queues `view` (a View) on `volume` (a VolumeRender); returns the ticket."""
        if out is None:
            out = np.empty((view.height, view.width, 4), np.float32)
        p, dev = _ptr(out)
        req = Request(volume._h, view, p, dev)
        t = C.c_uint64()
        _check(lib().mrp_serve_submit(self._h, C.byref(req), C.byref(t)))
        self._outs[t.value] = out
        return t.value

    def poll(self, ticket, wait_ms=-1):
        """(done, timing dict); raises MrpError if the request failed."""
        done = C.c_int()
        tm = RequestTiming()
        st = lib().mrp_serve_poll(self._h, ticket, int(wait_ms), C.byref(done), C.byref(tm))
        if done.value:
            out = self._outs.pop(ticket, None)
            _check(st)
            return True, {k: getattr(tm, k) for k, _ in RequestTiming._fields_}, out
        _check(st)
        return False, None, None

    def wait(self, ticket, timeout_s=300.0):
        """Blocks until done (at most timeout_s; None waits without a bound);
        returns (output, timing).  MrpError(ERR_TIMEOUT) when the bound ends
        first -- the request stays queued."""
        done, tm, out = self.poll(ticket, -1 if timeout_s is None else max(0, int(timeout_s * 1000)))
        if not done:
            raise MrpError(ERR_TIMEOUT, f"request {ticket} not done after {timeout_s} s")
        return out, tm

    def stats(self):
        st = ServeStats()
        _check(lib().mrp_serve_stats_get(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServeStats._fields_}

    def close(self):
        if self._h:
            _check(lib().mrp_serve_close(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Viewer:
    """The reference's real-time viewer loop, VolumeRender::Render(float3*
    target, Histogram*, unsigned* target2, ...) (core/volume.cu:550-628), over
    mrp_render_interactive: the running-mean image and the per-pixel
    histograms are device buffers (CUDA tensors) kept between frames; each
    frame returns the RGBA8 image ([H, W] uint32, 0xAARRGGBB)."""

    def __init__(self, volume, width, height, checkerboard=False):
        import torch
        self.volume, self.width, self.height = volume, int(width), int(height)
        self.target = torch.zeros((self.height, self.width, 3), dtype=torch.float32, device="cuda")
        self.histo = torch.zeros((self.height, self.width, 33), dtype=torch.float32, device="cuda")
        self.checkerboard = bool(checkerboard)
        self.frame_num = 0   # the reference's frameNum (reset when the camera moves)
        self.flip = 0
        self.rng_frame = 0   # randNum

    def reset(self):
        self.frame_num = 0

    def frame(self, view, rt, tone=2, denoise=False, exposure=1.0):
        view.width, view.height = self.width, self.height
        view.frame_offset = self.rng_frame
        out = np.empty((self.height, self.width), np.uint32)
        _check(lib().mrp_render_interactive(self.volume._h, C.byref(view), int(rt), self.frame_num,
                                            1 if self.checkerboard else 0, self.flip, int(tone),
                                            1 if denoise else 0, float(exposure), self.target.data_ptr(),
                                            self.histo.data_ptr(), out.ctypes.data, 0))
        self.frame_num += 1
        self.flip ^= 1
        self.rng_frame += 1
        return out
