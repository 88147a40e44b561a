"""The oracle's point, spot, directional and environment emitters (pointlight.cpp,
spotlight.cpp, directional.cpp, environment.cpp, distribution.cpp) pinned on the CPU:
direct lighting of the ground against closed-form irradiance, and the environment map's
importance sampling against its own pdf (the design of the reference's
environment_test.cpp: binned sample counts against the integrated pdf)."""
import math
import os

import numpy as np
import pytest

from gianduia_b200 import scenes
from oracle import pyoracle as O

ALBEDO = 0.6


def ground_direct(tmp_path, light):
    """One bounce (maxDepth 1) of the lights scene at 1 spp: the film holds exactly the
    next-event estimate of each camera sample. Returns (image, ground points, lit mask)."""
    W = H = 48
    xml = scenes.lights(str(tmp_path), width=W, height=H, spp=1, max_depth=1, emitters=(light,))
    sc = O.Scene.load(xml)
    film, _, _ = sc.render(0, 1)
    img = film[..., :3] / np.maximum(film[..., 3:4], 1e-9)
    py, px = np.mgrid[0:H, 0:W].astype(np.int32)
    rays = sc.camera_rays(0, px.ravel(), py.ravel())
    hit = sc.trace(rays)
    ground = hit["inst"] == 0
    t = np.where(ground, hit["t"], 0.0)   # misses have t = inf
    p = rays[:, 0:3] + rays[:, 4:7] * t[:, None]
    return sc, img.reshape(-1, 3), p, ground


def shadowed(sc, p, to_light, dist):
    r = np.zeros((p.shape[0], 8), np.float32)
    r[:, 0:3] = p
    r[:, 3] = 1e-4
    r[:, 4:7] = to_light
    r[:, 7] = dist - 1e-4
    occ, _, _ = sc.trace(r, anyhit=True)
    return occ


def test_point_light_irradiance(tmp_path):
    sc, img, p, ground = ground_direct(tmp_path, "point")
    props = scenes.LIGHTS["point"][1]
    pos, power = np.array(props["position"]), np.array(props["power"])
    d = pos - p
    dist = np.linalg.norm(d, axis=1)
    wi = d / dist[:, None]
    lit = ground & ~shadowed(sc, p, wi, dist)
    expect = (ALBEDO / math.pi) * power[None] / (4 * math.pi) * (wi[:, 1] / dist ** 2)[:, None]
    assert lit.sum() > 500
    assert np.allclose(img[lit], expect[lit], rtol=2e-5)
    assert (img[ground & ~lit] == 0).all()


def test_spot_light_cone(tmp_path):
    sc, img, p, ground = ground_direct(tmp_path, "spot")
    props = scenes.LIGHTS["spot"][1]
    pos, power = np.array(props["position"]), np.array(props["power"])
    axis = np.array(props["direction"]) / np.linalg.norm(props["direction"])
    half = props["spot_size"] * 0.5
    cos_total = math.cos(math.radians(half))
    cos_start = math.cos(math.radians(half * (1 - props["blend"])))
    d = pos - p
    dist = np.linalg.norm(d, axis=1)
    wi = d / dist[:, None]
    cos_t = -(wi @ axis)
    t = np.clip((cos_t - cos_total) / (cos_start - cos_total), 0, 1)
    falloff = np.where(cos_t <= cos_total, 0.0, np.where(cos_t < cos_start, t * t * (3 - 2 * t), 1.0))
    lit = ground & ~shadowed(sc, p, wi, dist)
    expect = (ALBEDO / math.pi) * power[None] / (4 * math.pi) * (falloff * wi[:, 1] / dist ** 2)[:, None]
    inside = lit & (falloff > 0)
    assert inside.sum() > 100 and (lit & (falloff == 0)).sum() > 50   # both sides of the cone edge
    assert np.allclose(img[lit], expect[lit], rtol=1e-4, atol=1e-6)


def test_directional_light(tmp_path):
    sc, img, p, ground = ground_direct(tmp_path, "directional")
    props = scenes.LIGHTS["directional"][1]
    wi = -np.array(props["direction"], np.float64)
    wi /= np.linalg.norm(wi)
    lit = ground & ~shadowed(sc, p, np.tile(wi, (p.shape[0], 1)), np.full(p.shape[0], 3e38))
    expect = (ALBEDO / math.pi) * np.array(props["irradiance"])[None] * wi[1]
    assert lit.sum() > 500
    assert np.allclose(img[lit], np.broadcast_to(expect, img[lit].shape), rtol=2e-5)


@pytest.fixture(scope="module")
def env(tmp_path_factory):
    d = tmp_path_factory.mktemp("env")
    path = os.path.join(str(d), "sky.exr")
    img = scenes.write_env_exr(path, width=32, height=16, sun=(0.3, 0.35), sun_size=0.08, sun_radiance=40.0)
    return O.EnvMap(path, strength=1.5), img


def test_env_pdf_normalised_and_sample_consistent(env):
    e, img = env
    rng = np.random.default_rng(1)
    n = 4000000   # the sun makes the pdf peaky: the Monte Carlo mean needs many samples
    z = 1 - 2 * rng.random(n)
    phi = 2 * np.pi * rng.random(n)
    s = np.sqrt(1 - z * z)
    dirs = np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)
    pdf = e.pdf(dirs)
    assert abs(pdf.mean() * 4 * np.pi - 1) < 0.01
    d, p, L = e.sample(rng.random((20000, 2)))
    ok = p > 0
    assert ok.mean() > 0.99
    # sample returns eval / pdf, and its pdf agrees with pdf() for the same direction
    assert np.allclose(L[ok] * p[ok, None], e.eval(d[ok]), rtol=1e-4, atol=1e-6)
    # (a direction that lands on a texel edge or at a pole may round into the neighbour)
    assert (np.abs(e.pdf(d[ok]) / p[ok] - 1) < 1e-3).mean() > 0.999
    # eval is strength x the bilinear image: at a texel centre, the texel itself
    v, u = 5, 20
    theta, ph = (v + 0.5) / 16 * np.pi, (u + 0.5) / 32 * 2 * np.pi
    w = np.array([[np.sin(theta) * np.cos(ph), np.sin(theta) * np.sin(ph), np.cos(theta)]])
    assert np.allclose(e.eval(w)[0], 1.5 * img[v, u], rtol=1e-4)


def test_env_sampling_histogram(env):
    """Sample counts per (theta, phi) bin against the pdf integrated over the bin."""
    e, _ = env
    rng = np.random.default_rng(2)
    bt, bp = 16, 32

    def bins(d):
        th = np.arccos(np.clip(d[:, 2], -1, 1))
        ph = np.arctan2(d[:, 1], d[:, 0]) % (2 * np.pi)
        return np.clip((th / np.pi * bt).astype(int), 0, bt - 1) * bp + np.clip((ph / (2 * np.pi) * bp).astype(int), 0, bp - 1)

    m = 1000000
    z = 1 - 2 * rng.random(m)
    phi = 2 * np.pi * rng.random(m)
    s = np.sqrt(1 - z * z)
    dirs = np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)
    expected = np.bincount(bins(dirs), weights=e.pdf(dirs) * 4 * np.pi / m, minlength=bt * bp)
    expected /= expected.sum()
    n = 300000
    d, p, _ = e.sample(rng.random((n, 2)))
    observed = np.bincount(bins(d[p > 0]), minlength=bt * bp)
    exp_n = expected * observed.sum()
    keep = exp_n > 20
    chi2 = float(((observed[keep] - exp_n[keep]) ** 2 / exp_n[keep]).sum())
    dof = int(keep.sum()) - 1
    # chi-square with ~500 degrees of freedom: mean dof, sd sqrt(2 dof); the pdf side is
    # itself a Monte Carlo estimate, so allow a wide margin
    assert chi2 < dof + 8 * np.sqrt(2 * dof) + 0.02 * dof, (chi2, dof)
    # the sun holds a large share of both
    assert observed[expected.argmax()] > 0.5 * exp_n[expected.argmax()]
