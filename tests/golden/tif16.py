"""Minimal reader of baseline little-endian 16-bit grayscale TIFFs (one
image, uncompressed, any number of strips): the images the reference and
this project write.  Returns rows in file order (the writers store them
bottom-up)."""
import struct

import numpy as np


def read_tif16(path):
    b = open(path, "rb").read()
    assert b[:4] == b"II*\x00", "not a little-endian TIFF"
    ifd = struct.unpack_from("<I", b, 4)[0]
    n = struct.unpack_from("<H", b, ifd)[0]
    tags = {}
    for k in range(n):
        tag, typ, count, value = struct.unpack_from("<HHII", b, ifd + 2 + 12 * k)
        if typ == 3 and count == 1:
            value &= 0xFFFF
        tags[tag] = (typ, count, value)

    def values(tag):
        typ, count, value = tags[tag]
        size = {3: 2, 4: 4}[typ]
        if count * size <= 4:
            raw = struct.pack("<I", value)[:count * size]
        else:
            raw = b[value:value + count * size]
        return list(struct.unpack("<%d%s" % (count, "H" if typ == 3 else "I"), raw))

    width, length = values(256)[0], values(257)[0]
    assert values(258)[0] == 16
    offs, counts = values(273), values(279)
    data = b"".join(b[o:o + c] for o, c in zip(offs, counts))
    return np.frombuffer(data[:2 * width * length], dtype="<u2").reshape(length, width)
