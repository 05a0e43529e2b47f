"""The default colour wheel of FlowToColor: the reference's 256x256 RGBA table, byte for byte.

The reference embeds the table in its library (src/colorwheel.cpp, COLOR_WHEEL_D,
include/flowfilter/colorwheel.h:20-27) and FlowToColor looks every pixel up in it; the colours
are not reproducible from a formula, so the table is data that has to be the same.  It is kept
here as ``colorwheel.z``: the rows delta-coded along x (each byte minus its left neighbour,
modulo 256, per channel) and zlib-compressed.  The library embeds the decoded table at build
time.

    python colorwheel_asset.py extract <reference src/colorwheel.cpp> colorwheel.z
        reads the table from the reference source and writes the asset
    python colorwheel_asset.py emit colorwheel.z <out.cpp>
        writes the C++ source of the table that the Makefile compiles into libffb200.so
"""

from __future__ import annotations

import hashlib
import re
import sys
import zlib

import numpy as np

SIZE = 256 * 256 * 4
# sha256 of the 262,144 table bytes (row-major, RGBA)
SHA256 = "966163576b67b0a8dfee44fd06e692f64572f7c92291fb4c2eae56c353ddea03"


def decode(blob: bytes) -> np.ndarray:
    d = np.frombuffer(zlib.decompress(blob), np.uint8)
    if d.size != SIZE:
        raise ValueError("colour wheel asset has the wrong size")
    return np.cumsum(d.reshape(256, 256, 4), axis=1, dtype=np.uint64).astype(np.uint8)


def encode(table: np.ndarray) -> bytes:
    t = np.ascontiguousarray(table, dtype=np.uint8).reshape(256, 256, 4)
    d = np.diff(t.astype(np.int16), axis=1, prepend=0).astype(np.uint8)
    return zlib.compress(d.tobytes(), 9)


def load(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        return decode(f.read())


def extract(ref_cpp: str) -> np.ndarray:
    src = open(ref_cpp).read()
    body = src[src.index("COLOR_WHEEL_D[]"):]
    vals = [int(x, 16) for x in re.findall(r"0x([0-9A-Fa-f]{2})", body)]
    if len(vals) != SIZE:
        raise ValueError(f"expected {SIZE} table bytes, found {len(vals)}")
    return np.array(vals, np.uint8).reshape(256, 256, 4)


def emit(table: np.ndarray, out_cpp: str) -> None:
    b = np.ascontiguousarray(table, dtype=np.uint8).tobytes()
    lines = [", ".join(str(v) for v in b[i:i + 32]) for i in range(0, len(b), 32)]
    with open(out_cpp, "w") as f:
        f.write("// generated by colorwheel_asset.py from colorwheel.z: the default colour wheel\n")
        f.write("extern const unsigned char ffb_colorwheel_rgba[%d];\n" % SIZE)
        f.write("const unsigned char ffb_colorwheel_rgba[%d] = {\n" % SIZE)
        f.write(",\n".join(lines))
        f.write("};\n")


def main() -> None:
    if len(sys.argv) != 4 or sys.argv[1] not in ("extract", "emit"):
        sys.exit(__doc__)
    if sys.argv[1] == "extract":
        t = extract(sys.argv[2])
        with open(sys.argv[3], "wb") as f:
            f.write(encode(t))
        print(hashlib.sha256(t.tobytes()).hexdigest())
    else:
        t = load(sys.argv[2])
        if hashlib.sha256(t.tobytes()).hexdigest() != SHA256:
            sys.exit("colour wheel asset: checksum mismatch")
        emit(t, sys.argv[3])


if __name__ == "__main__":
    main()
