"""Build ``mrpnn_model.bin``: the MRPNN network weights plus the stencil directions.

The trained network of the reference ships as ``training_pipeline/NNWeight.npy``
(146 named fp32 arrays, identical to the ``__constant__`` / ``__device__`` arrays
of ``core/NNWeight.cuh``).  Its feature stencil uses 160 fixed unit directions
(``Spn0..Spn4``, ``SpVn5..SpVn7`` in ``core/vector.cu:82-177``) that the weights
were trained against, so they are part of the model, not of the renderer.  This
script packs both into one little-endian file::

    b"MRPNNMD1", u32 n_tensors,
    n_tensors x { u16 name_len, name (ascii), u32 count, f32[count] }

with the stencil directions stored as tensor ``STENCIL_DIRS`` (160 x 3, index
order of ``SphereRandom3``) and the digit permutations of the scrambled radical
inverse that the HG lookup table integrates with (``RadicalInversePermutations_``
in ``core/volume.cu:1195``, the 2 + 3 + 5 + 7 + 11 = 28 entries of bases 2-11,
the only bases Fill_Hg uses) as tensor ``HALTON_PERMS`` (28 values).  The LUT
the network was trained with was built from that table, so it is model data.
It cross-checks every weight array against the ``.cuh`` copy before writing.

Usage: python make_model.py /path/to/reference [out.bin]
"""
import os
import re
import struct
import sys

import numpy as np

TABLES = ["Spn0", "Spn1", "Spn2", "Spn3", "Spn4", "SpVn5", "SpVn6", "SpVn7"]
TABLE_SIZES = [8, 8, 16, 16, 16, 32, 32, 32]


def parse_cuh_arrays(text):
    out = {}
    for m in re.finditer(r"float\s+(\w+)\[(\d+)\]\s*=\s*\{([^}]*)\}", text):
        vals = np.array([float(v) for v in m.group(3).replace("\n", "").split(",") if v.strip()],
                        dtype=np.float32)
        if vals.size != int(m.group(2)):
            raise ValueError(f"{m.group(1)}: {vals.size} values, declared {m.group(2)}")
        out[m.group(1)] = vals
    return out


def parse_stencil(text):
    dirs = []
    for name, n in zip(TABLES, TABLE_SIZES):
        m = re.search(r"float3\s+" + name + r"\[(\d+)\]\s*=\s*\{(.*?)\};", text, re.S)
        if not m or int(m.group(1)) != n:
            raise ValueError(f"stencil table {name} not found")
        trip = re.findall(r"float3\{([^}]*)\}", m.group(2))
        vals = [[float(c) for c in t.split(",")] for t in trip]
        if len(vals) != n:
            raise ValueError(f"{name}: {len(vals)} entries")
        dirs.extend(vals)
    return np.asarray(dirs, dtype=np.float32)


HALTON_BASES = (2, 3, 5, 7, 11)


def parse_halton_perms(text):
    m = re.search(r"RadicalInversePermutations_\[\]\s*=\s*\{([^}]*)\}", text)
    if not m:
        raise ValueError("RadicalInversePermutations_ not found")
    vals = [int(v) for v in m.group(1).replace("\n", "").split(",") if v.strip()]
    perms = np.asarray(vals[:sum(HALTON_BASES)], dtype=np.float32)
    off = 0
    for b in HALTON_BASES:   # each base's block is a permutation of its digits
        if sorted(perms[off:off + b].astype(int)) != list(range(b)):
            raise ValueError(f"base {b}: not a permutation")
        off += b
    return perms


def build(ref_root, out_path):
    weights = np.load(os.path.join(ref_root, "training_pipeline", "NNWeight.npy"),
                      allow_pickle=True).item()
    with open(os.path.join(ref_root, "core", "NNWeight.cuh")) as f:
        cuh = parse_cuh_arrays(f.read())
    if set(cuh) != set(weights):
        raise ValueError("NNWeight.npy and NNWeight.cuh disagree on names")
    for k, v in weights.items():
        if not np.array_equal(np.asarray(v, dtype=np.float32).ravel(), cuh[k]):
            raise ValueError(f"{k}: npy and cuh values differ")
    with open(os.path.join(ref_root, "core", "vector.cu")) as f:
        dirs = parse_stencil(f.read())
    tensors = [(k, np.asarray(weights[k], dtype=np.float32).ravel()) for k in sorted(weights)]
    tensors.append(("STENCIL_DIRS", dirs.ravel()))
    with open(os.path.join(ref_root, "core", "volume.cu")) as f:
        tensors.append(("HALTON_PERMS", parse_halton_perms(f.read())))
    with open(out_path, "wb") as f:
        f.write(b"MRPNNMD1")
        f.write(struct.pack("<I", len(tensors)))
        for name, arr in tensors:
            nb = name.encode("ascii")
            f.write(struct.pack("<H", len(nb)))
            f.write(nb)
            f.write(struct.pack("<I", arr.size))
            f.write(arr.astype("<f4").tobytes())
    return out_path


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    out = sys.argv[2] if len(sys.argv) > 2 else os.path.join(os.path.dirname(__file__), "mrpnn_model.bin")
    print(build(ref, out))
