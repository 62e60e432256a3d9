"""mrpnn_b200 -- B200-native (sm_100a) MRPNN render path: delta-tracking path
tracer and the MRPNN neural radiance predictor, behind a C ABI
(include/mrpnn.h) with a Python mirror of the reference's VolumeRender /
Camera API."""
from .api import (BF16, FP8, FP32, NOALLOC_MAX_POINTS, Camera, MrpError, Server, Viewer, VolumeRender, camera_frame,
                  debug_alloc_calls, default_params, hg_lut_lookup, read_hdri, init, lib, predict_features, predict_features_noalloc, read_volume_file,
                  write_volume_bin)

__all__ = ["VolumeRender", "Camera", "MrpError", "init", "lib", "predict_features", "predict_features_noalloc",
           "NOALLOC_MAX_POINTS", "debug_alloc_calls", "hg_lut_lookup", "read_hdri", "Server", "Viewer", "read_volume_file", "write_volume_bin", "camera_frame", "default_params", "FP32", "BF16", "FP8"]
