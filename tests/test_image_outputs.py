"""Image outputs on the CPU: the PNG / EXR writers (read back with independent readers),
and the oracle's post-processing restatement (tonemap.frag, bloom_*.frag,
gammaCorrect.frag, Film::savePNG) pinned against formulas written out here in float64
numpy from the same shader text."""
import numpy as np
import pytest

import gianduia_b200 as G
from oracle import pyoracle as O

from imagefiles import read_exr, read_png


def test_png_round_trip(tmp_path):
    img = (np.random.default_rng(1).random((37, 53, 3)) * 256).astype(np.uint8)
    G.write_png(str(tmp_path / "a.png"), img)
    assert np.array_equal(read_png(str(tmp_path / "a.png")), img)


def test_exr_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    img = (rng.standard_normal((29, 41, 3)) * 10).astype(np.float32)
    img[0, 0] = [np.inf, -0.0, 1e-40]
    G.write_exr(str(tmp_path / "a.exr"), img)
    back, attrs = read_exr(str(tmp_path / "a.exr"))
    assert np.array_equal(back.view(np.uint32), img.view(np.uint32))
    assert attrs["lineOrder"][1] == b"\x00" and attrs["pixelAspectRatio"][0] == "float"


def test_writers_reject_bad_arguments(tmp_path):
    with pytest.raises(G.GndError):
        G.write_png(str(tmp_path / "no_such_dir" / "a.png"), np.zeros((2, 2, 3), np.uint8))
    with pytest.raises(G.GndError):
        G.write_exr(str(tmp_path / "b.exr"), np.zeros((0, 2, 3), np.float32))


# ---------------------------------------------------------------- tonemap operators, float64
def srgb_export(x):
    s = np.where(x <= 0.0031308, 12.92 * x, 1.055 * np.power(np.maximum(x, 0), 1 / 2.4) - 0.055)
    return np.clip(s * 255 + 0.5, 0, 255).astype(np.uint8)


def mat(m):   # GLSL column-major mat3 -> row-major numpy
    return np.array(m, np.float64).reshape(3, 3).T


def reinhard(c):
    luma = c @ [0.2126, 0.7152, 0.0722]
    return c * ((luma / (1 + luma)) / np.maximum(luma, 1e-5))[..., None]


def uncharted2(c):
    A, B, C, D, E, F = 0.15, 0.5, 0.1, 0.2, 0.02, 0.3
    f = lambda x: ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - E / F
    return f(2 * c) / f(11.2)


def aces(c):
    i = mat([0.59719, 0.07600, 0.02840, 0.35458, 0.90834, 0.13383, 0.04823, 0.01566, 0.83777])
    o = mat([1.60475, -0.10208, -0.00327, -0.53108, 1.10813, -0.07276, -0.07367, -0.00605, 1.07602])
    v = c @ i.T
    v = (v * (v + 0.0245786) - 0.000090537) / (v * (0.983729 * v + 0.432951) + 0.238081)
    return np.clip(v @ o.T, 0, 1)


def khronos(c):
    sc, ds = 0.8 - 0.04, 0.15
    x = c.min(axis=-1)
    c = c - np.where(x < 0.08, x - 6.25 * x * x, 0.04)[..., None]
    peak = c.max(axis=-1)
    d = 1 - sc
    npk = 1 - d * d / (peak + d - sc)
    g = 1 - 1 / (ds * (peak - npk) + 1)
    out = c * (npk / peak)[..., None] * (1 - g)[..., None] + (npk * g)[..., None]
    return np.where((peak < sc)[..., None], c, out)


def agx(c, power, sat):
    to2020 = mat([0.6274, 0.0691, 0.0164, 0.3293, 0.9195, 0.0880, 0.0433, 0.0113, 0.8956])
    from2020 = mat([1.6605, -0.1246, -0.0182, -0.5876, 1.1329, -0.1006, -0.0728, -0.0083, 1.1187])
    inset = mat([0.856627153315983, 0.137318972929847, 0.11189821299995, 0.0951212405381588, 0.761241990602591,
                 0.0767994186031903, 0.0482516061458583, 0.101439036467562, 0.811302368396859])
    outset = mat([1.1271005818144368, -0.1413297634984383, -0.14132976349843826, -0.11060664309660323,
                  1.157823702216272, -0.11060664309660294, -0.016493938717834573, -0.016493938717834257,
                  1.2519364065950405])
    lo, hi = -12.47393, 4.026069
    v = np.maximum(c @ to2020.T @ inset.T, 1e-10)
    v = np.clip((np.clip(np.log2(v), lo, hi) - lo) / (hi - lo), 0, 1)
    x2, x4 = v * v, v ** 4
    v = 15.5 * x4 * x2 - 40.14 * x4 * v + 31.96 * x4 - 6.868 * x2 * v + 0.4298 * x2 + 0.1191 * v - 0.00232
    v = np.sign(v) * np.abs(v) ** power if power == 1.0 else np.power(v, power)
    luma = v @ [0.2126, 0.7152, 0.0722]
    v = luma[..., None] + sat * (v - luma[..., None])
    v = np.power(np.maximum(v @ outset.T, 0), 2.2)
    return np.clip(v @ from2020.T, 0, 1)


OPS = {0: lambda c: c, 1: reinhard, 2: uncharted2, 3: aces, 4: khronos, 5: lambda c: agx(c, 1.0, 1.0),
       6: lambda c: agx(c, 1.35, 1.4)}


@pytest.mark.parametrize("op", sorted(OPS))
def test_oracle_tonemap_operators(op):
    rng = np.random.default_rng(op)
    img = (rng.random((24, 31, 3)) ** 3 * 20).astype(np.float32)
    hdr, b8 = O.post(img, tonemapper=op, exposure=0.5)
    ref = OPS[op](img.astype(np.float64) * 2 ** 0.5)
    ok = np.isfinite(ref)
    # AgX's sixth-degree polynomial cancels: float32 evaluation is good to ~1e-4 there
    tol = 1e-4 if op >= 5 else 2e-5
    assert np.allclose(hdr[ok], ref[ok], rtol=tol, atol=tol / 10), np.abs(hdr - ref)[ok].max()
    # Film::savePNG conversion: within one level where float32 rounding meets a boundary
    d = np.abs(b8.astype(int) - srgb_export(np.where(ok, ref, 0)).astype(int))
    assert d.max() <= 1 and (d == 0).mean() > 0.99


def test_oracle_display_gamma():
    img = np.linspace(0, 1.2, 3 * 40 * 3, dtype=np.float32).reshape(3, 40, 3)
    _, b8 = O.post(img, output=1)
    s = np.where(img <= 0.0031308, 12.92 * img.astype(np.float64), 1.055 * np.power(img.astype(np.float64), 0.41666) - 0.055)
    ref = np.rint(np.clip(s, 0, 1) * 255)
    assert np.abs(b8.astype(int) - ref.astype(int)).max() <= 1


def test_oracle_bloom_properties():
    rng = np.random.default_rng(7)
    img = (rng.random((64, 96, 3)) * 0.5).astype(np.float32)
    base, _ = O.post(img)
    # nothing above the threshold: the bloom adds nothing
    same, _ = O.post(img, bloom=True, threshold=1.0)
    assert np.array_equal(same, base)
    # one bright block: light spreads around it and only adds
    img2 = img.copy()
    img2[30:34, 46:50] = 40.0
    b0, _ = O.post(img2)
    b1, _ = O.post(img2, bloom=True, threshold=1.0, intensity=0.04)
    add = b1 - b0
    assert (add >= -1e-6).all() and add[20:44, 36:60].sum() > 0.5 * add.sum()
    assert add[32, 40].sum() > add[32, 10].sum() >= 0.0
    # fewer mips spread less far
    b2, _ = O.post(img2, bloom=True, threshold=1.0, intensity=0.04, mips=2)
    assert (b2 - b0)[:, :20].sum() < add[:, :20].sum()


def test_half_rounding_matches_ieee():
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.standard_normal(3000) * 10.0 ** rng.integers(-8, 5, 3000),
                        [65504, 65519.9, 65520, 2 ** -24, 3 * 2 ** -26, 0.0]]).astype(np.float32)
    ours = np.array([O.round_half(float(v)) for v in x], np.float32)
    with np.errstate(over="ignore"):
        assert np.array_equal(ours, x.astype(np.float16).astype(np.float32))


# ---------------------------------------------------------------- OpenEXR reader
def exr_bytes(img, compression, half=False, extra_channel=False):
    """An OpenEXR file written here from the format specification: scanline blocks of 1
    (none, ZIPS) or 16 (ZIP) lines; ZIP blocks reordered (even bytes, then odd) and delta
    coded before zlib."""
    import struct
    import zlib
    h, w, _ = img.shape
    names = [b"A", b"B", b"G", b"R"] if extra_channel else [b"B", b"G", b"R"]
    ptype = 1 if half else 2
    hdr = bytearray(struct.pack("<II", 20000630, 2))

    def attr(name, typ, value):
        hdr.extend(name + b"\0" + typ + b"\0" + struct.pack("<i", len(value)) + value)

    attr(b"channels", b"chlist", b"".join(n + b"\0" + struct.pack("<iBBBBii", ptype, 0, 0, 0, 0, 1, 1) for n in names) + b"\0")
    attr(b"compression", b"compression", bytes([compression]))
    box = struct.pack("<iiii", 0, 0, w - 1, h - 1)
    attr(b"dataWindow", b"box2i", box)
    attr(b"displayWindow", b"box2i", box)
    attr(b"lineOrder", b"lineOrder", b"\0")
    attr(b"pixelAspectRatio", b"float", struct.pack("<f", 1.0))
    attr(b"screenWindowCenter", b"v2f", struct.pack("<ff", 0, 0))
    attr(b"screenWindowWidth", b"float", struct.pack("<f", 1.0))
    hdr.extend(b"\0")
    dt = "<f2" if half else "<f4"
    chan = {b"R": 0, b"G": 1, b"B": 2}
    per = 16 if compression == 3 else 1
    blocks = []
    for y0 in range(0, h, per):
        raw = b""
        for y in range(y0, min(h, y0 + per)):
            for n in names:
                vals = img[y, :, chan[n]] if n in chan else np.full(w, 0.5)
                raw += vals.astype(dt).tobytes()
        data = raw
        if compression in (2, 3):
            r = np.frombuffer(raw, np.uint8)
            t = np.concatenate([r[0::2], r[1::2]])
            d = t.astype(np.int32).copy()
            d[1:] = (t[1:].astype(np.int32) - t[:-1].astype(np.int32) + 128) & 255
            data = zlib.compress(d.astype(np.uint8).tobytes())
        blocks.append(struct.pack("<ii", y0, len(data)) + data)
    table, off = b"", len(hdr) + 8 * len(blocks)
    for b in blocks:
        table += struct.pack("<Q", off)
        off += len(b)
    return bytes(hdr) + table + b"".join(blocks)


@pytest.mark.parametrize("compression,half,extra", [(0, False, False), (2, False, False), (3, False, True),
                                                    (3, True, False), (0, True, True)])
def test_exr_reader(tmp_path, compression, half, extra):
    rng = np.random.default_rng(compression * 10 + half)
    img = (rng.random((37, 21, 3)) * 8).astype(np.float32)
    if half:
        img = img.astype(np.float16).astype(np.float32)
    p = tmp_path / "in.exr"
    p.write_bytes(exr_bytes(img, compression, half, extra))
    assert np.array_equal(G.read_exr(str(p)), img)


def test_exr_reader_round_trip_and_errors(tmp_path):
    img = np.random.default_rng(5).random((9, 13, 3)).astype(np.float32)
    G.write_exr(str(tmp_path / "a.exr"), img)
    assert np.array_equal(G.read_exr(str(tmp_path / "a.exr")), img)
    (tmp_path / "bad.exr").write_bytes(b"not an exr file at all")
    with pytest.raises(G.GndError):
        G.read_exr(str(tmp_path / "bad.exr"))
    with pytest.raises(G.GndError):
        G.read_exr(str(tmp_path / "missing.exr"))
