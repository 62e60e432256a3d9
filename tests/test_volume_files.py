"""Volume files of the reference (LoadData, core/volume.cu:970-1149) read by
the library's host code: the .bin cache format, .txt and .vox.  No GPU."""
import numpy as np
import pytest


def test_bin_round_trip(tmp_path):
    import mrpnn_b200 as M
    R = 12
    rng = np.random.default_rng(0)
    data = rng.uniform(-0.5, 2.0, (R, R, R)).astype(np.float32)   # negative = SDF distance, kept
    p = str(tmp_path / "cloud.bin")
    M.write_volume_bin(p, data)
    raw = open(p, "rb").read()
    assert np.frombuffer(raw[:4], np.int32)[0] == R and len(raw) == 4 + 4 * R ** 3
    np.testing.assert_array_equal(np.frombuffer(raw[4:], np.float32).reshape(R, R, R), data)
    np.testing.assert_array_equal(M.read_volume_file(p), data)


def test_txt_and_bin_cache(tmp_path):
    import mrpnn_b200 as M
    R = 6
    data = (np.arange(R ** 3, dtype=np.float32) / 7.0).reshape(R, R, R)
    p = tmp_path / "vol.txt"
    flat = data.ravel()
    with open(p, "w") as f:
        f.write(f"{R}\n")
        for i in range(0, flat.size, 8):
            f.write(" ".join(f"{x:.9g}" for x in flat[i:i + 8]) + "\n")
    np.testing.assert_array_equal(M.read_volume_file(str(p)), data)
    # a .bin written beside it is preferred (the reference's cache)
    M.write_volume_bin(str(p) + ".bin", data * 2)
    np.testing.assert_array_equal(M.read_volume_file(str(p)), data * 2)


def test_vox(tmp_path):
    import mrpnn_b200 as M
    rng = np.random.default_rng(1)
    ints = rng.integers(0, 256, 256 ** 3)
    p = tmp_path / "model.vox"
    with open(p, "w") as f:
        f.write("w 256\nh 256\nd 256\n")
        rows = ints.reshape(-1, 64)
        f.write("\n".join(" ".join(map(str, r)) for r in rows))
        f.write("\n")
    got = M.read_volume_file(str(p))
    np.testing.assert_allclose(got.ravel(), ints.astype(np.float32) * np.float32(64.0 / 255.0), rtol=1e-7)


def test_bad_files(tmp_path):
    import mrpnn_b200 as M
    with pytest.raises(M.MrpError):
        M.read_volume_file(str(tmp_path / "missing.bin"))
    p = tmp_path / "short.bin"
    p.write_bytes(np.array([8], np.int32).tobytes() + np.zeros(10, np.float32).tobytes())
    with pytest.raises(M.MrpError, match="truncated"):
        M.read_volume_file(str(p))
    q = tmp_path / "x.raw"
    q.write_bytes(b"abc")
    with pytest.raises(M.MrpError, match="not a .bin"):
        M.read_volume_file(str(q))
