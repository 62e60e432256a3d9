"""The C ABI without a GPU: the library loads, exports every symbol that
include/mrpnn.h declares, and refuses to run (no CPU fallback)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(mrp_[a-z0-9_]+)\s*\(", text))
    return names - {"mrp_fill_fn"}


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"mrp_init", "mrp_volume_create", "mrp_volume_update", "mrp_render", "mrp_predict_features"} <= names


def test_library_exports_every_declared_symbol():
    import mrpnn_b200
    L = mrpnn_b200.lib()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(L, n)]
    assert not missing, missing
    from mrpnn_b200 import api
    assert set(api._SIGS) == declared_symbols()


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="a GPU is present")
def test_fails_loudly_without_gpu():
    import mrpnn_b200
    from mrpnn_b200 import api
    with pytest.raises(mrpnn_b200.MrpError) as e:
        mrpnn_b200.init()
    assert e.value.status == api.ERR_NO_DEVICE
    with pytest.raises(mrpnn_b200.MrpError):
        mrpnn_b200.predict_features(np.zeros((1, 576), np.float32), np.zeros(1, np.float32), 0.5, (1, 1, 1))
    import ctypes as C
    h = C.c_void_p()
    assert api.lib().mrp_volume_create_ex(64, 1, C.byref(h)) == api.ERR_NOT_READY   # fp16 grid
    assert api.lib().mrp_render_wait(None, 0) == api.ERR_NOT_READY
    with pytest.raises(mrpnn_b200.MrpError):
        mrpnn_b200.VolumeRender(64, storage="fp16")


def test_grid_storage_names():
    import mrpnn_b200
    from mrpnn_b200 import api
    assert api.STORAGE == {"fp32": 0, "fp16": 1}
    with pytest.raises(ValueError):
        mrpnn_b200.VolumeRender(64, storage="bf16")   # rejected before any device call


def test_default_params():
    import mrpnn_b200
    p = mrpnn_b200.default_params()
    assert list(p.scatter_rate) == pytest.approx([1.001] * 3)
    assert p.bake_res == 768 and p.tr_scale == 1.0 and p.precision == 0


def test_serve_defaults_and_no_gpu_refusal():
    import ctypes as C
    import mrpnn_b200
    from mrpnn_b200 import api
    cfg = api.ServeConfig()
    api.lib().mrp_serve_default_config(C.byref(cfg))
    assert cfg.memory_budget == 120 << 30 and cfg.max_slots == 16 and cfg.precision == api.BF16
    assert cfg.slot_pixels == 0
    p = mrpnn_b200.default_params()
    assert p.nee_mode == 0
    if not _has_gpu():
        h = C.c_void_p()
        assert api.lib().mrp_serve_open(C.byref(cfg), C.byref(h)) == api.ERR_NOT_READY


def test_model_file_layout():
    """The packed model file holds the 146 reference tensors plus the stencil."""
    import struct
    path = os.path.join(ROOT, "mrpnn_b200", "data", "mrpnn_model.bin")
    with open(path, "rb") as f:
        assert f.read(8) == b"MRPNNMD1"
        n = struct.unpack("<I", f.read(4))[0]
        total = 0
        names = []
        for _ in range(n):
            ln = struct.unpack("<H", f.read(2))[0]
            names.append(f.read(ln).decode())
            c = struct.unpack("<I", f.read(4))[0]
            f.seek(4 * c, 1)
            total += c if names[-1] not in ("STENCIL_DIRS", "HALTON_PERMS") else 0
    assert n == 148 and "STENCIL_DIRS" in names and "HALTON_PERMS" in names
    assert total == 49673


def test_header_is_plain_c(tmp_path):
    """include/mrpnn.h is a C99 header (the FFI boundary): a C program that
    calls entry points links against the library."""
    import shutil
    import subprocess
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else shutil.which("gcc")
    if not cc:
        pytest.skip("no C compiler")
    src = tmp_path / "abi.c"
    src.write_text('#include "mrpnn.h"\n'
                   "int main(void) {\n"
                   "    mrp_volume* v = 0;\n"
                   "    mrp_params p;\n"
                   "    mrp_default_params(&p);\n"
                   "    if (mrp_volume_create_ex(8, MRP_STORAGE_FP16, &v) == MRP_OK) return 1;  /* no device here */\n"
                   "    return mrp_render_wait(v, 0) == MRP_OK;\n"
                   "}\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib = os.path.join(root, "mrpnn_b200")
    exe = tmp_path / "abi"
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I" + os.path.join(root, "include"),
                    "-I/usr/local/cuda/include", str(src), "-o", str(exe), "-L" + lib, "-lmrpnn_b200",
                    "-Wl,-rpath," + lib], check=True)
    if not _has_gpu():
        assert subprocess.run([str(exe)]).returncode == 0


def test_feature_sets_are_validated_before_the_c_abi():
    """The predictor entry points read n * 576 and n floats from the caller's
    pointers; malformed arrays are refused in the host mirror with a clear
    error, before any device or C ABI call."""
    import mrpnn_b200
    good_f, good_g = np.zeros((3, 576), np.float32), np.zeros(3, np.float32)
    for fn in (mrpnn_b200.predict_features, mrpnn_b200.predict_features_noalloc):
        with pytest.raises(ValueError, match="576"):
            fn(np.zeros((3, 575), np.float32), good_g, 0.5, (1, 1, 1))
        with pytest.raises(ValueError, match="576"):
            fn(np.zeros(576, np.float32), np.zeros(1, np.float32), 0.5, (1, 1, 1))
        with pytest.raises(ValueError, match="gamma"):
            fn(good_f, np.zeros(4, np.float32), 0.5, (1, 1, 1))
    with pytest.raises(ValueError, match="out"):
        mrpnn_b200.predict_features(good_f, good_g, 0.5, (1, 1, 1), out=np.zeros((3, 4), np.float32))


def test_allocation_counter_needs_no_device():
    import mrpnn_b200
    assert isinstance(mrpnn_b200.debug_alloc_calls(), int)
