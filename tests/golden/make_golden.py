"""Convert the reference's BSON golden fields into compressed .npz fixtures.

The reference pins its 2D solver with three final-pressure fields written by
ReferenceTests.jl/BSON.jl (test/references/acoustic2D_*.bson, produced by
test/test2D_xPU.jl:108-195). Julia is not available here, so this script parses
the BSON bytes directly and stores each field as a float64 array in Julia's
column-major order, i.e. ``pend[i, j]`` of the reference is ``arr[i, j]`` of the
.npz after ``np.asfortranarray``. Values are copied bit for bit.

Run once where the reference tree is mounted:

    python tests/golden/make_golden.py /path/to/AcousticWaveCPML.jl

The .npz files it writes are committed; nothing at test time reads the
reference tree.
"""
import os
import struct
import sys

import numpy as np

CASES = (
    "acoustic2D_center_halo20",
    "acoustic2D_center_freetop_halo20",
    "acoustic2D_gradient_freetop_halo20",
)


def _cstring(buf, pos):
    end = buf.index(b"\x00", pos)
    return buf[pos:end].decode(), end + 1


def parse_bson(buf, pos=0):
    """Minimal BSON document parser covering the element types BSON.jl emits
    for a Float64 array: document (0x03), array (0x04), string (0x02),
    binary (0x05), int64 (0x12), int32 (0x10) and double (0x01)."""
    (size,) = struct.unpack_from("<i", buf, pos)
    end = pos + size - 1
    pos += 4
    out = {}
    while pos < end:
        etype = buf[pos]
        pos += 1
        key, pos = _cstring(buf, pos)
        if etype in (0x03, 0x04):
            (sub,) = struct.unpack_from("<i", buf, pos)
            val = parse_bson(buf, pos)
            if etype == 0x04:
                val = [val[k] for k in sorted(val, key=int)]
            pos += sub
        elif etype == 0x02:
            (n,) = struct.unpack_from("<i", buf, pos)
            val = buf[pos + 4 : pos + 4 + n - 1].decode()
            pos += 4 + n
        elif etype == 0x05:
            (n,) = struct.unpack_from("<i", buf, pos)
            val = bytes(buf[pos + 5 : pos + 5 + n])
            pos += 5 + n
        elif etype == 0x12:
            (val,) = struct.unpack_from("<q", buf, pos)
            pos += 8
        elif etype == 0x10:
            (val,) = struct.unpack_from("<i", buf, pos)
            pos += 4
        elif etype == 0x01:
            (val,) = struct.unpack_from("<d", buf, pos)
            pos += 8
        else:
            raise ValueError(f"unsupported BSON element type 0x{etype:02x}")
        out[key] = val
    return out


def load_julia_array(path, key="pend"):
    doc = parse_bson(open(path, "rb").read())
    node = doc[key]
    assert node["tag"] == "array", node["tag"]
    assert node["type"]["name"] == ["Core", "Float64"], node["type"]
    shape = tuple(node["size"])
    flat = np.frombuffer(node["data"], dtype="<f8")
    assert flat.size == int(np.prod(shape))
    return np.asfortranarray(flat.reshape(shape, order="F"))


def main(ref_root):
    here = os.path.dirname(os.path.abspath(__file__))
    for name in CASES:
        src = os.path.join(ref_root, "test", "references", name + ".bson")
        arr = load_julia_array(src)
        dst = os.path.join(here, name + ".npz")
        np.savez_compressed(dst, pend=arr)
        print(f"{name}: shape={arr.shape} absmax={np.abs(arr).max():.4e} -> {dst}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <root of the AcousticWaveCPML.jl source tree>")
    main(sys.argv[1])
