"""The oracle's procedural and image textures (math/perlin.h, math/worley.h,
textures/perlin.h, marble.h, wood.h, cellular.h, domainWarp.h, imageTexture.cpp,
textureCache.h) against float32 numpy restatements written from the same formulas:
Perlin noise and turbulence, Worley F1/F2 in three metrics, the texture blends, the domain
warp's shift of p and uv, and image lookups (closest / bilinear, repeat / clamp, sRGB
decode, vertical flip, 16-bit PNG to 8 bits, EXR through half precision)."""
import os

import numpy as np
import pytest

from gianduia_b200 import scenes
from oracle import pyoracle as O

F = np.float32


def _xml(tmp_path, body, name="tex.xml"):
    path = os.path.join(str(tmp_path), name)
    with open(path, "w") as f:
        f.write(body + "\n")
    return path


# ---------------------------------------------------------------- restatements
PERM = None


def perm():
    global PERM
    if PERM is None:
        PERM = O.perlin_perm().astype(np.int64)
    return PERM


def fade(t):
    return t * t * t * (t * (t * F(6) - F(15)) + F(10))


def grad(h, x, y, z):
    h = h & 15
    u = np.where(h < 8, x, y)
    v = np.where(h < 4, y, np.where((h == 12) | (h == 14), x, z))
    return np.where(h & 1, -u, u) + np.where(h & 2, -v, v)


def lerp(t, a, b):
    return (F(1) - t) * a + t * b


def noise(p):
    P = perm()
    fl = np.floor(p)
    X, Y, Z = [(fl[:, k].astype(np.int64) & 255) for k in range(3)]
    x, y, z = [p[:, k] - fl[:, k] for k in range(3)]
    u, v, w = fade(x), fade(y), fade(z)
    A = P[X] + Y
    AA, AB = P[A] + Z, P[A + 1] + Z
    B = P[X + 1] + Y
    BA, BB = P[B] + Z, P[B + 1] + Z
    one = F(1)
    g000 = grad(P[AA], x, y, z)
    g100 = grad(P[BA], x - one, y, z)
    g010 = grad(P[AB], x, y - one, z)
    g110 = grad(P[BB], x - one, y - one, z)
    g001 = grad(P[AA + 1], x, y, z - one)
    g101 = grad(P[BA + 1], x - one, y, z - one)
    g011 = grad(P[AB + 1], x, y - one, z - one)
    g111 = grad(P[BB + 1], x - one, y - one, z - one)
    y0 = lerp(v, lerp(u, g000, g100), lerp(u, g010, g110))
    y1 = lerp(v, lerp(u, g001, g101), lerp(u, g011, g111))
    return lerp(w, y0, y1)


def turbulence(p, octaves):
    acc = np.zeros(p.shape[0], F)
    weight = F(1)
    t = p.copy()
    for _ in range(octaves):
        acc = acc + weight * np.abs(noise(t))
        weight = weight * F(0.5)
        t = t * F(2)
    return np.clip(acc, F(0), F(1))


def worley(p, metric):
    def hash1(n):
        n = ((n << np.uint32(13)) ^ n).astype(np.uint32)
        n = (n * (n * n * np.uint32(15731) + np.uint32(789221)) + np.uint32(1376312589)).astype(np.uint32)
        return (n & np.uint32(0x7FFFFFFF)).astype(F) / F(0x7FFFFFFF)

    base = np.floor(p).astype(np.int64)
    f1 = np.full(p.shape[0], F(1e8))
    f2 = np.full(p.shape[0], F(1e8))
    with np.errstate(over="ignore"):
        for k in (-1, 0, 1):
            for j in (-1, 0, 1):
                for i in (-1, 0, 1):
                    c = base + np.array([i, j, k])
                    cu = c.astype(np.int32).view(np.uint32)
                    n = (cu[:, 0] * np.uint32(73856093)) ^ (cu[:, 1] * np.uint32(19349663)) ^ (cu[:, 2] * np.uint32(83492791))
                    fp = c.astype(F) + np.stack([hash1(n), hash1(n + np.uint32(1)), hash1(n + np.uint32(2))], axis=1)
                    d = p - fp
                    if metric == 0:
                        dist = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
                    elif metric == 1:
                        dist = np.abs(d[:, 0]) + np.abs(d[:, 1]) + np.abs(d[:, 2])
                    else:
                        dist = np.max(np.abs(d), axis=1)
                    closer = dist < f1
                    second = ~closer & (dist < f2)
                    f2 = np.where(closer, f1, np.where(second, dist, f2))
                    f1 = np.where(closer, dist, f1)
    return f1, f2


def mix(t, a, b):
    return np.asarray(a, F)[None, :] * (F(1) - t)[:, None] + np.asarray(b, F)[None, :] * t[:, None]


def points(n, seed, lo=-4.0, hi=4.0):
    return np.random.default_rng(seed).uniform(lo, hi, (n, 3)).astype(F)


# ---------------------------------------------------------------- tests
def test_permutation_table():
    P = perm()
    assert sorted(P[:256]) == list(range(256))
    assert np.array_equal(P[:256], P[256:])
    assert list(P[:6]) == [151, 160, 137, 91, 90, 15]


def test_noise_zero_on_lattice_and_bounded(tmp_path):
    x = _xml(tmp_path, scenes._texture("perlin_color", "t", {"scale": 1.0, "octaves": 1}))
    lattice = np.random.default_rng(1).integers(-50, 50, (500, 3)).astype(F)
    assert np.all(O.tex_eval(x, lattice) == 0.0)
    assert np.all(np.abs(noise(points(20000, 2, -100, 100))) <= 1.0)


@pytest.mark.parametrize("octaves,scale", [(1, 1.0), (5, 0.35), (8, 2.5)])
def test_perlin_texture(tmp_path, octaves, scale):
    v1, v2 = (0.2, 0.25, 0.3), (0.8, 0.75, 0.6)
    x = _xml(tmp_path, scenes._texture("perlin_color", "t", {"value1": v1, "value2": v2, "scale": scale, "octaves": octaves}))
    p = points(4000, octaves)
    got = O.tex_eval(x, p)
    want = mix(turbulence(p / F(scale), octaves), v1, v2)
    assert np.abs(got - want).max() <= 1e-6


def test_perlin_defaults(tmp_path):
    """value1 0, value2 1, scale 1, octaves 6 (perlin.h:15-27)."""
    x = _xml(tmp_path, '<texture type="perlin_color"/>')
    p = points(2000, 3)
    t = turbulence(p, 6)
    assert np.abs(O.tex_eval(x, p) - t[:, None]).max() <= 1e-6


@pytest.mark.parametrize("kind", ["marble", "wood"])
def test_marble_wood(tmp_path, kind):
    props = {"scale": 0.4, "octaves": 4, "vein_freq": 7.0, "turb_scale": 3.0, "axis": (0.3, 1.0, 0.2)}
    x = _xml(tmp_path, scenes._texture(kind + "_color", "t", props))
    p = points(4000, 5, -2, 2)
    axis = np.array(props["axis"], np.float64)
    axis = (axis / np.linalg.norm(axis)).astype(F)
    turb = turbulence(p / F(0.4), 4)
    if kind == "marble":
        val = (p @ axis.astype(np.float64)).astype(F) + turb * F(3)
        t = F(0.5) * (F(1) + np.sin(val * F(7)))
        v1, v2 = (0.1, 0.1, 0.1), (0.9, 0.9, 0.9)
    else:
        radius = np.linalg.norm(np.cross(p.astype(np.float64), axis.astype(np.float64)), axis=1).astype(F) + turb * F(3)
        t = np.abs(np.sin(radius * F(7)))
        v1, v2 = (0.6, 0.4, 0.2), (0.3, 0.15, 0.05)
    got = O.tex_eval(x, p)
    want = mix(t, v1, v2)
    # the dot / cross products are restated in float64 here: a few ulp of their argument,
    # times the vein frequency, through sin
    assert np.abs(got - want).max() <= 2e-5


@pytest.mark.parametrize("mode", ["distance", "cracks"])
@pytest.mark.parametrize("metric", ["euclidean", "manhattan", "chebyshev"])
def test_cellular(tmp_path, mode, metric):
    v1, v2 = (0.1, 0.2, 0.3), (0.9, 0.8, 0.7)
    x = _xml(tmp_path, scenes._texture("cellular_color", "t", {"value1": v1, "value2": v2, "scale": 0.5, "mode": mode, "metric": metric}))
    p = points(3000, 9, -20, 20)
    f1, f2 = worley(p / F(0.5), ["euclidean", "manhattan", "chebyshev"].index(metric))
    n = np.clip(f2 - f1 if mode == "cracks" else f1, F(0), F(1))
    want = np.asarray(v1, F)[None, :] * (F(1) - n)[:, None] + np.asarray(v2, F)[None, :] * n[:, None]
    assert np.abs(O.tex_eval(x, p) - want).max() <= 1e-6


def test_cellular_unknown_names_fall_back(tmp_path):
    """cellular.h:27-44: unknown mode -> distance, unknown metric -> euclidean."""
    a = _xml(tmp_path, scenes._texture("cellular_color", "t", {"mode": "bogus", "metric": "bogus"}), "a.xml")
    b = _xml(tmp_path, scenes._texture("cellular_color", "t", {}), "b.xml")
    p = points(500, 4)
    assert np.array_equal(O.tex_eval(a, p), O.tex_eval(b, p))


def test_domain_warp(tmp_path):
    """domainWarp.h:38-58: p moves by (2 w - 1) strength; uv by its projections on dpdu and
    n x dpdu; the base texture is evaluated there."""
    base = scenes._texture("checkerboard_color", "base", {"value1": (1, 1, 1), "value2": (0, 0, 0), "scale": (0.1, 0.1)})
    warp = scenes._texture("perlin_color", "warp", {"scale": 0.7, "octaves": 3})
    x = _xml(tmp_path, scenes._texture("domainWarp_color", "t", {"strength": 0.3}, [base, warp]))
    rng = np.random.default_rng(3)
    p = points(3000, 6, -2, 2)
    n = rng.normal(size=(3000, 3))
    n = (n / np.linalg.norm(n, axis=1, keepdims=True)).astype(F)
    dpdu = np.cross(n, rng.normal(size=(3000, 3))).astype(F) * F(1.5)
    dpdu[:10] = 0.0
    uv = rng.uniform(-1, 1, (3000, 2)).astype(F)
    got = O.tex_eval(x, p, n, dpdu, uv)
    w = turbulence(p / F(0.7), 3)
    d = (w * F(2) - F(1)) * F(0.3)
    dvec = np.stack([d, d, d], axis=1)
    dpdv = np.cross(n.astype(np.float64), dpdu.astype(np.float64))
    lu = np.sum(dpdu.astype(np.float64) ** 2, axis=1)
    lv = np.sum(dpdv ** 2, axis=1)
    du = np.where(lu > 0, np.sum(dvec * dpdu, axis=1) / np.where(lu > 0, lu, 1), 0)
    dv = np.where(lv > 0, np.sum(dvec * dpdv, axis=1) / np.where(lv > 0, lv, 1), 0)
    u2, v2 = uv[:, 0] + du, uv[:, 1] + dv
    s = np.floor(u2 / 0.1).astype(np.int64) + np.floor(v2 / 0.1).astype(np.int64)
    want = np.where(s % 2 == 0, 1.0, 0.0)
    # squares whose edge lies within float rounding of the warped uv may differ
    edge = (np.abs(u2 / 0.1 - np.round(u2 / 0.1)) < 1e-4) | (np.abs(v2 / 0.1 - np.round(v2 / 0.1)) < 1e-4)
    assert np.mean(got[~edge, 0] == want[~edge]) == 1.0
    assert np.all(got[:10, 0] == np.where((np.floor(uv[:10, 0] / F(0.1)).astype(int) + np.floor(uv[:10, 1] / F(0.1)).astype(int)) % 2 == 0, 1, 0))


def test_domain_warp_needs_both_children(tmp_path):
    base = scenes._texture("checkerboard_color", "base", {})
    x = _xml(tmp_path, scenes._texture("domainWarp_color", "t", {}, [base]))
    with pytest.raises(RuntimeError, match="warp"):
        O.tex_eval(x, points(1, 0))


def _image_lookup(data, uv, linear, clamp):
    """imageTexture.cpp:84-143 on an [h, w, c] float32 array (row 0 = the image's bottom)."""
    h, w, c = data.shape
    if clamp:
        lu = np.clip(uv, F(0), F(1))
    else:
        lu = uv - np.floor(uv)

    def at(x, y):
        if clamp:
            x, y = np.clip(x, 0, w - 1), np.clip(y, 0, h - 1)
        else:
            x, y = x % w, y % h
        v = data[y, x]
        return v[:, :3] if c >= 3 else np.repeat(v[:, :1], 3, axis=1)

    if not linear:
        return at(np.floor(lu[:, 0] * F(w)).astype(np.int64), np.floor(lu[:, 1] * F(h)).astype(np.int64))
    xc = lu[:, 0] * F(w) - F(0.5)
    yc = lu[:, 1] * F(h) - F(0.5)
    x0, y0 = np.floor(xc).astype(np.int64), np.floor(yc).astype(np.int64)
    tx = (xc - x0.astype(F))[:, None]
    ty = (yc - y0.astype(F))[:, None]
    top = at(x0, y0) * (F(1) - tx) + at(x0 + 1, y0) * tx
    bot = at(x0, y0 + 1) * (F(1) - tx) + at(x0 + 1, y0 + 1) * tx
    return top * (F(1) - ty) + bot * ty


def _srgb(v):
    v = v.astype(F)
    return np.where(v <= F(0.04045), v / F(12.92), ((v + F(0.055)) / F(1.055)).astype(np.float64) ** 2.4).astype(F)


@pytest.mark.parametrize("channels", [1, 2, 3, 4])
@pytest.mark.parametrize("mode", ["closest-repeat", "linear-repeat", "linear-clamp", "closest-clamp"])
def test_png_texture(tmp_path, channels, mode):
    rng = np.random.default_rng(channels)
    img = rng.integers(0, 256, (9, 13, channels)).astype(np.uint8)
    scenes.write_png(str(tmp_path / "t.png"), img)
    linear, clamp = mode.startswith("linear"), mode.endswith("clamp")
    x = _xml(tmp_path, scenes._texture("image_color", "t", {
        "filename": "t.png", "interpolation_mode": "linear" if linear else "closest",
        "repeat_mode": "clamp" if clamp else "repeat", "color_space": "sRGB"}))
    uv = rng.uniform(-1.5, 2.5, (4000, 2)).astype(F)
    got = O.tex_eval(x, np.zeros((4000, 3), F), uv=uv)
    data = img[::-1].astype(F) / F(255)
    # textureCache.h:80-84: every channel of 1-3 channel images, RGB of RGBA images
    dec = _srgb(data)
    if channels == 4:
        dec[..., 3] = data[..., 3]
    want = _image_lookup(dec, uv, linear, clamp)
    # the sRGB curve's pow is float here and float64 in the restatement
    assert np.abs(got - want).max() <= 2e-6


def test_png_16bit_keeps_high_byte(tmp_path):
    rng = np.random.default_rng(5)
    img = rng.integers(0, 65536, (6, 7, 3)).astype(np.uint16)
    scenes.write_png(str(tmp_path / "t.png"), img)
    x = _xml(tmp_path, scenes._texture("image_color", "t", {"filename": "t.png"}))
    uv = (np.stack(np.meshgrid(np.arange(7) + 0.5, np.arange(6) + 0.5), axis=-1).reshape(-1, 2) / [7, 6]).astype(F)
    got = O.tex_eval(x, np.zeros((42, 3), F), uv=uv)
    want = (img[::-1] >> 8).astype(F).reshape(-1, 3) / F(255)
    assert np.array_equal(got, want)


def test_exr_texture_goes_through_half(tmp_path):
    rng = np.random.default_rng(8)
    rgb = (rng.random((5, 6, 3)) * 3).astype(F)
    scenes.write_exr_float(str(tmp_path / "t.exr"), rgb)
    x = _xml(tmp_path, scenes._texture("image_color", "t", {"filename": "t.exr", "interpolation_mode": "linear"}))
    uv = rng.uniform(0, 1, (3000, 2)).astype(F)
    got = O.tex_eval(x, np.zeros((3000, 3), F), uv=uv)
    half = rgb.astype(np.float16).astype(F)[::-1]
    want = _image_lookup(np.concatenate([half, np.ones((5, 6, 1), F)], axis=-1), uv, True, False)
    assert np.array_equal(got, want)
    assert not np.array_equal(half, rgb[::-1])


def test_image_texture_bad_options(tmp_path):
    scenes.write_png(str(tmp_path / "t.png"), np.zeros((2, 2, 3), np.uint8))
    for prop, msg in [("interpolation_mode", "interpolation"), ("color_space", "color space"), ("repeat_mode", "repeat")]:
        x = _xml(tmp_path, scenes._texture("image_color", "t", {"filename": "t.png", prop: "bogus"}))
        with pytest.raises(RuntimeError, match=msg):
            O.tex_eval(x, points(1, 0))
