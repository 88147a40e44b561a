"""The film's reconstruction filters on the GPU against the oracle, above all the
reference's default: a scene without <filter> gets a Gaussian of radius 2 and alpha 2
(film.cpp:29, filter.h:34-54), which spreads every sample over up to 16 pixels
(film.h:26-69).

  * same stream: the default Gaussian and an explicit one (radius (1.5, 1.0), alpha 3)
    through path and volpath: per-pixel weight sums agree to float rounding (the weights
    go through expf on the device and std::exp on the host) and the images meet the
    same-stream bar of the other image tests;
  * batched equals plain: bit-identical sum wL and sum w (fixed-point film);
  * statistics with independent seeds: a Gaussian film correlates neighbouring pixels and
    its per-pixel sum of w L^2 does not give a standard error, so K independent renders
    per side give per-pixel means and standard errors; the fraction of pixel channels
    beyond 3 combined standard errors must stay under a binomial bound around the rate a
    t distribution with 2(K - 1) degrees of freedom gives (failures listed)."""
import math

import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O
from test_gpu_render import image, same_stream_check
from statbounds import binomial_bound, t_tail

pytestmark = pytest.mark.gpu

FILTERS = {"default": "default", "explicit": ("gaussian", (1.5, 1.0), 3.0)}


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("scene", ["cornell", "volumetric"])
@pytest.mark.parametrize("filt", sorted(FILTERS))
def test_gaussian_same_stream(ctx, tmp_path, scene, filt):
    gen = scenes.cornell if scene == "cornell" else scenes.volumetric
    xml = gen(str(tmp_path), width=64, height=48, spp=4, max_depth=8, filter=FILTERS[filt])
    hs = G.HostScene.load_xml(xml)
    assert hs.desc.filter == 1
    sid = ctx.upload(hs)
    gfilm, st = ctx.render(sid, spp=4)
    ofilm, paths, _ = O.Scene.load(xml).render(0, 4)
    assert st["paths"] == paths == 64 * 48 * 4
    # the weights: same sample positions, the same filter formula
    np.testing.assert_allclose(gfilm[..., 3], ofilm[..., 3], rtol=2e-6, atol=1e-6)
    assert float(gfilm[..., 3].min()) > 0.0
    same_stream_check(image(gfilm), image(ofilm), "%s-%s" % (scene, filt), min_frac=0.995)
    ctx.free_scene(sid)


@pytest.mark.parametrize("filt", sorted(FILTERS))
def test_gaussian_batched_equals_plain(ctx, tmp_path, filt):
    """Batched renders gather the film from per-sample records (kFilmFromSamplesGauss),
    plain ones splat with atomics: the fixed-point sums must agree bit for bit, also for a
    pixel window whose samples reach pixels outside it."""
    xml = scenes.cornell(str(tmp_path), width=40, height=30, spp=6, filter=FILTERS[filt])
    sid = ctx.upload(G.HostScene.load_xml(xml))
    a, _ = ctx.render(sid, spp=6)
    b, _ = ctx.render(sid, spp=6, batched=True)
    assert np.array_equal(a[..., :4], b[..., :4])
    np.testing.assert_allclose(a[..., 4:], b[..., 4:], rtol=1e-5, atol=1e-6)
    wa, _ = ctx.render(sid, spp=3, window=(7, 5, 23, 19))
    wb, _ = ctx.render(sid, spp=3, window=(7, 5, 23, 19), batched=True)
    assert np.array_equal(wa[..., :4], wb[..., :4])
    assert wa[:3].sum() == 0 and wa[:, :5].sum() == 0 and wa[:, 25:].sum() == 0   # at most 2 pixels past the window
    if filt == "default":
        assert wa[4, 6:24, 3].min() > 0   # the row above the window gets weight
    ctx.free_scene(sid)


def batch_sigma_check(g_imgs, o_imgs, label):
    """Per-pixel 3-sigma agreement from K independent images per side: returns the count of
    channels beyond 3 combined standard errors and its bound."""
    g, o = np.stack(g_imgs), np.stack(o_imgs)
    K = g.shape[0]
    mg, mo = g.mean(axis=0), o.mean(axis=0)
    se = np.sqrt(g.var(axis=0, ddof=1) / K + o.var(axis=0, ddof=1) / K)
    valid = se > 1e-9
    z = np.abs(mg - mo) / np.maximum(se, 1e-12)
    beyond = (z > 3) & valid
    n = int(valid.sum())
    p = t_tail(3.0, 2 * (K - 1))
    bound = binomial_bound(n, p)
    worst = np.argsort(-np.where(valid, z, 0).ravel())[:8]
    listed = [(np.unravel_index(int(i), z.shape), round(float(z.ravel()[i]), 2)) for i in worst]
    assert int(beyond.sum()) <= bound, "%s: %d of %d channels beyond 3 sigma (bound %d, expected %.1f): %s" % (
        label, int(beyond.sum()), n, bound, n * p, listed)
    return int(beyond.sum()), bound


@pytest.mark.parametrize("scene", ["cornell", "volumetric"])
def test_gaussian_statistics(ctx, tmp_path, scene):
    K, spp = 16, 8
    gen = scenes.cornell if scene == "cornell" else scenes.volumetric
    xml = gen(str(tmp_path), width=32, height=32, spp=spp, max_depth=8, filter="default")
    sid = ctx.upload(G.HostScene.load_xml(xml))
    osc = O.Scene.load(xml)
    g = [image(ctx.render(sid, spp=spp, first_pass=200000 + k * spp, batched=True)[0]) for k in range(K)]
    o = [image(osc.render(k * spp, (k + 1) * spp)[0]) for k in range(K)]
    batch_sigma_check(g, o, "%s-gaussian-%dx%d" % (scene, K, spp))
    ctx.free_scene(sid)
