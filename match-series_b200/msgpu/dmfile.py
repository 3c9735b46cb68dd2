"""Writer of Gatan DigitalMicrograph 3/4 files (the public tag-tree format):
synthetic DM images for tests and benchmarks of the DM3/DM4 reader.

Layout: big-endian header (version, length, byte order 1), a root tag
directory whose entries are directories (identifier 20) or tags (21); a tag is
"%%%%", an info count and info words (32-bit in version 3, 64-bit in
version 4, big-endian) followed by little-endian values.  Each image is an
entry of ImageList with ImageData.Data (an array), ImageData.DataType and
ImageData.Dimensions (nameless entries 0, 1).  Unrelated tags (a group, an
array of groups, a string) are added around it, as real files carry them.
"""
from __future__ import annotations

import struct

import numpy as np

DTYPES = {2: "<i2", 3: "<i4", 4: "<u2", 5: "<u4", 6: "<f4", 7: "<f8", 10: "<u1"}


class _W:
    def __init__(self, version: int):
        self.v = version
        self.out = bytearray()

    def word(self, x: int):
        self.out += struct.pack(">i" if self.v == 3 else ">q", x)

    def name(self, ident: int, name: str):
        nb = name.encode()
        self.out += struct.pack(">Bh", ident, len(nb)) + nb
        if self.v == 4:
            self.out += struct.pack(">q", 0)

    def tag(self, name: str, info, payload: bytes):
        self.name(21, name)
        self.out += b"%%%%"
        self.word(len(info))
        for x in info:
            self.word(x)
        self.out += payload

    def directory(self, name: str, entries):
        self.name(20, name)
        self.out += bytes([1, 0])
        self.word(len(entries))
        for e in entries:
            e(self)


def _value(t: int, x) -> bytes:
    return np.array([x], dtype=DTYPES[t]).tobytes()


def dm_bytes(images, version: int = 3) -> bytes:
    """images: list of (array (ny, nx), type code); the reader takes the last."""
    w = _W(version)
    w.out += struct.pack(">i", version)
    w.word(0)                        # file length (not used by readers here)
    w.out += struct.pack(">i", 1)    # little-endian values
    w.out += bytes([1, 0])

    def filler(x):
        x.tag("Filler", [15, 0, 2, 0, 2, 0, 6], _value(2, -3) + _value(6, 1.5))

    def thumbs(x):
        x.tag("Thumbnails", [20, 15, 0, 2, 0, 3, 0, 3, 2],
              _value(3, 1) + _value(3, 2) + _value(3, 3) + _value(3, 4))

    def image_entry(arr, t):
        ny, nx = arr.shape
        data = np.ascontiguousarray(arr, dtype=DTYPES[t]).tobytes()

        def ent(x):
            image_data = [lambda y: y.tag("Data", [20, t, nx * ny], data),
                          lambda y: y.tag("DataType", [5], _value(5, t)),
                          lambda y: y.directory("Dimensions", [lambda z: z.tag("", [5], _value(5, nx)),
                                                               lambda z: z.tag("", [5], _value(5, ny))])]
            name = "frame".encode("utf-16-le")
            x.directory("", [lambda y: y.tag("Name", [20, 4, len(name) // 2], name),
                             lambda y: y.directory("ImageData", image_data),
                             lambda y: y.tag("UniqueID", [5], _value(5, 7))])
        return ent

    root = [filler, lambda x: x.directory("ImageList", [image_entry(a, t) for a, t in images]), thumbs]
    w.word(len(root))
    for e in root:
        e(w)
    w.out += bytes(8)
    return bytes(w.out)
