"""Radiance .hdr environment maps (VolumeRender::SetHDRI, core/volume.cu:
1696-1728): the library's reader (mrp_hdri_file_read, host only) against
the reference's own loader (core/hdr_loader.h, compiled on the CPU) on
files written here -- flat and run-length encoded scanlines, flat lines
inside an encoded file, the small-exponent quirk of the RGBE conversion,
header variants -- and the errors on malformed files."""
import os

import numpy as np
import pytest

from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference checker not available")


def _rle_component(vals):
    """New-style RLE of one component: runs of >= 3 equal bytes, literals."""
    out, i, n = bytearray(), 0, len(vals)
    while i < n:
        j = i
        while j < n and j - i < 127 and vals[j] == vals[i]:
            j += 1
        if j - i >= 3:
            out += bytes([128 + (j - i), vals[i]])
            i = j
            continue
        k = i
        while k < n and k - i < 128:
            if k + 2 < n and vals[k] == vals[k + 1] == vals[k + 2]:
                break
            k += 1
        out += bytes([k - i]) + bytes(vals[i:k])
        i = k
    return bytes(out)


def write_hdr(path, rgbe, mode="rle", header=("FORMAT=32-bit_rle_rgbe",), flat_rows=()):
    """rgbe: uint8 [h, w, 4].  mode: "rle" (every row encoded unless listed in
    flat_rows) or "flat"."""
    h, w, _ = rgbe.shape
    with open(path, "wb") as f:
        f.write(b"#?RADIANCE\n")
        for line in header:
            f.write(line.encode() + b"\n")
        f.write(b"\n")
        f.write(f"-Y {h} +X {w}\n".encode())
        for j in range(h):
            row = rgbe[j]
            if mode == "flat" or j in flat_rows:
                f.write(row.tobytes())
            else:
                f.write(bytes([2, 2, w >> 8, w & 255]))
                for c in range(4):
                    f.write(_rle_component(list(row[:, c])))


def _random_rgbe(rng, h, w, runs=True):
    px = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    px[..., 3] = rng.integers(120, 140, (h, w))
    if runs:   # long runs for the encoder
        px[:, w // 4: w // 2, :] = px[:, w // 4: w // 4 + 1, :]
    px[0, :3, 3] = [0, 1, 5]   # black, and exponents below 9 (the conversion's bit quirk)
    return px


def _product(path):
    import mrpnn_b200 as M
    return M.read_hdri(path)


@needs_ref
@pytest.mark.parametrize("case", ["rle", "flat_small", "flat_wide", "mixed", "two_prefix", "header"])
def test_reader_matches_reference(tmp_path, case):
    rng = np.random.default_rng(sum(map(ord, case)))
    p = str(tmp_path / f"{case}.hdr")
    if case == "rle":
        write_hdr(p, _random_rgbe(rng, 6, 40))
    elif case == "flat_small":          # width < 8: never run-length encoded
        write_hdr(p, _random_rgbe(rng, 4, 5, runs=False), mode="flat")
    elif case == "flat_wide":           # an encodable width written flat
        px = _random_rgbe(rng, 3, 33)
        px[:, 0, 0] = 7                 # a flat line must not start with byte 2
        write_hdr(p, px, mode="flat")
    elif case == "mixed":               # flat rows inside an encoded file
        px = _random_rgbe(rng, 5, 24)
        px[:, 0, 0] = 9
        write_hdr(p, px, flat_rows=(1, 3))
    elif case == "two_prefix":          # a flat row whose first pixel is (2, g != 2, ...)
        px = _random_rgbe(rng, 3, 16)
        px[1, 0, :] = [2, 7, 40, 130]
        write_hdr(p, px, flat_rows=(1,))
    else:                               # comments, exposure and gamma lines, xyze format
        write_hdr(p, _random_rgbe(rng, 2, 12), header=("# made by a test", "EXPOSURE=2.5", "GAMMA=2.2",
                                                         "FORMAT=32-bit_rle_xyze", "SOFTWARE=none"))
    ref = O.ref_load_hdr(p)
    assert ref is not None
    got = _product(p)
    np.testing.assert_array_equal(got, ref)
    assert (got[..., 3] == 0).all()


@needs_ref
@pytest.mark.parametrize("case", ["format", "truncated", "length", "nores"])
def test_reader_refuses_what_the_reference_refuses(tmp_path, case):
    import mrpnn_b200 as M
    rng = np.random.default_rng(5)
    p = str(tmp_path / f"bad_{case}.hdr")
    if case == "format":
        write_hdr(p, _random_rgbe(rng, 2, 10), header=("FORMAT=32-bit_rle_float",))
    elif case == "truncated":
        write_hdr(p, _random_rgbe(rng, 4, 20))
        with open(p, "rb+") as f:
            f.truncate(os.path.getsize(p) - 10)
    elif case == "length":              # encoded length differs from the width
        px = _random_rgbe(rng, 2, 20)
        write_hdr(p, px)
        data = bytearray(open(p, "rb").read())
        k = data.index(bytes([2, 2, 0, 20]))
        data[k + 3] = 21
        open(p, "wb").write(bytes(data))
    else:                               # no resolution line before the end
        with open(p, "wb") as f:
            f.write(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n")
    if case != "nores":                 # the reference's reader dereferences NULL at end of file
        assert O.ref_load_hdr(p) is None
    with pytest.raises(M.MrpError):
        M.read_hdri(p)


def test_reader_known_values(tmp_path):
    """(m + 0.5) * 2^(e - 136): RGBE (128, 64, 0, 129) is (1.00391, 0.50391, 0.00391)."""
    p = str(tmp_path / "one.hdr")
    px = np.zeros((1, 3, 4), np.uint8)
    px[0, 0] = [128, 64, 0, 129]
    px[0, 1] = [255, 255, 255, 0]       # exponent 0: black
    px[0, 2] = [10, 20, 30, 136]
    write_hdr(p, px, mode="flat")
    got = _product(p)[0]
    np.testing.assert_array_equal(got[0], np.float32([128.5 / 128, 64.5 / 128, 0.5 / 128, 0]))
    np.testing.assert_array_equal(got[1], np.zeros(4, np.float32))
    np.testing.assert_array_equal(got[2], np.float32([10.5, 20.5, 30.5, 0]))


def test_set_hdri_needs_a_device():
    from mrpnn_b200 import api
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    m = np.zeros((2, 4, 4), np.float32)
    assert api.lib().mrp_volume_set_hdri(None, m.ctypes.data, 4, 2) == api.ERR_NOT_READY
    assert api.lib().mrp_volume_load_hdri(None, b"x.hdr") != api.OK
