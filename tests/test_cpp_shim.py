"""The C++ drop-in (include/mrpnn_volume_render.hpp): builds on the CPU, and
on the GPU renders the reference README's example through the reference's
class API, matching the same frame rendered through the Python ABI mirror."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "shim_example.cpp")


def build(tmp):
    exe = os.path.join(tmp, "shim_example")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    lib = os.path.join(ROOT, "mrpnn_b200")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", SRC,
                    "-o", exe, "-L" + lib, "-lmrpnn_b200", "-Wl,-rpath," + lib, "-pthread"], check=True)
    return exe


def test_shim_builds(tmp_path):
    assert os.path.exists(build(str(tmp_path)))


@pytest.mark.gpu
def test_shim_renders_like_python_api(tmp_path):
    exe = build(str(tmp_path))
    prefix = str(tmp_path / "frame")
    r = subprocess.run([exe, prefix], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert os.path.getsize(prefix + ".png") > 100
    img = np.fromfile(prefix + ".f32", np.float32).reshape(64, 64, 4)
    import mrpnn_b200 as M
    v = M.VolumeRender(64)
    v.SetDatas(lambda x, y, z, u, w, t: (np.sqrt((u - .5) ** 2 + (w - .5) ** 2 + (t - .5) ** 2) < 0.25).astype(np.float32))
    v.Update()
    v.SetScatterRate(0.99)
    L = np.array([0.3, 0.8, 0.5], np.float32)
    L /= np.float32(np.sqrt(np.float32(np.dot(L, L))))
    ori, up, right = M.camera_frame((0.75, 0.75, 0.75))
    ref = v.Render((64, 64), ori, up, right, L, M.VolumeRender.MRPNN, 0.857, 8.0, (1, 1, 1), 1, 2)
    assert (img[..., 3] > 0).sum() > 100
    np.testing.assert_allclose(img, ref, rtol=1e-5, atol=1e-6)
    img16 = np.fromfile(prefix + ".fp16.f32", np.float32).reshape(64, 64, 4)
    np.testing.assert_array_equal(img16.view(np.uint32), img.view(np.uint32))
