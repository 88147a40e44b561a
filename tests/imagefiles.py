"""Minimal readers for the image files gnd_image_write_png / gnd_image_write_exr write,
written from the file format specifications (PNG: chunks with CRC-32, zlib stream of
filtered scanlines; OpenEXR: magic, version, attribute header, line offset table,
uncompressed scanline blocks), so that the tests check the files independently of the
writer."""
import struct
import zlib

import numpy as np


def read_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n", "not a PNG file"
    pos, chunks = 8, []
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        typ = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(typ + body) & 0xFFFFFFFF == crc, "bad CRC in %r" % typ
        chunks.append((typ, body))
        pos += 12 + n
    assert chunks[0][0] == b"IHDR" and chunks[-1][0] == b"IEND"
    w, h, depth, ctype, comp, filt, inter = struct.unpack(">IIBBBBB", chunks[0][1])
    assert (depth, ctype, comp, filt, inter) == (8, 2, 0, 0, 0)
    raw = zlib.decompress(b"".join(b for t, b in chunks if t == b"IDAT"))
    rows = np.frombuffer(raw, np.uint8).reshape(h, 3 * w + 1)
    assert (rows[:, 0] == 0).all(), "only filter type 0 is written"
    return rows[:, 1:].reshape(h, w, 3).copy()


def read_exr(path):
    data = open(path, "rb").read()
    magic, version = struct.unpack("<II", data[:8])
    assert magic == 20000630 and version == 2
    pos, attrs = 8, {}
    while data[pos] != 0:
        end = data.index(b"\0", pos)
        name = data[pos:end].decode()
        tend = data.index(b"\0", end + 1)
        typ = data[end + 1:tend].decode()
        n, = struct.unpack("<i", data[tend + 1:tend + 5])
        attrs[name] = (typ, data[tend + 5:tend + 5 + n])
        pos = tend + 5 + n
    pos += 1
    # channels
    typ, ch = attrs["channels"]
    assert typ == "chlist"
    names, p = [], 0
    while ch[p] != 0:
        end = ch.index(b"\0", p)
        names.append(ch[p:end].decode())
        ptype, = struct.unpack("<i", ch[end + 1:end + 5])
        assert ptype == 2, "FLOAT channels"
        p = end + 17
    assert attrs["compression"][1] == b"\x00"
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    offsets = struct.unpack("<%dQ" % h, data[pos:pos + 8 * h])
    img = np.zeros((h, w, len(names)), np.float32)
    for off in offsets:
        y, nbytes = struct.unpack("<ii", data[off:off + 8])
        line = np.frombuffer(data[off + 8:off + 8 + nbytes], "<f4").reshape(len(names), w)
        img[y - y0] = line.T
    order = [names.index(c) for c in "RGB"]
    return img[..., order], attrs
