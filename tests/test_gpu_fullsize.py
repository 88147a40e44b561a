"""Parity at the benchmark configurations' full sizes.

  * microfacet grid (5,242,882 triangles, 4105 instances, 1024 x 1024): one pass on the
    same per-pixel streams as the CPU oracle (same-stream bar of test_gpu_render), and
    per-pixel 3-sigma agreement with independent seeds at 256 x 256, 16 spp;
  * Cornell box at its benchmark size (256 x 256, 16 spp) and the volumetric Cornell box
    at its resolution and depth (512 x 512, depth 32, 2 passes) on the oracle's streams;
  * size-independent properties at the full sample counts: the batched engine and the
    plain engine give bit-identical film sums for the microfacet render (1024^2 x 64 spp)
    and the volumetric Cornell box (512^2 x 64 spp, depth 32), every sample lands in the
    film once (total weight = samples, up to the rare samples on a pixel border that the
    box filter gives to two pixels), and the radiance is finite and non-negative."""
import os

import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O
from test_gpu_render import image, same_stream_check, sigma_check

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(900)]


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def microfacet_xml(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("microfacet"))
    return scenes.microfacet(d, width=1024, height=1024, spp=64, max_depth=16, grid=64, seed=2)


def check_film(f, samples, label):
    assert np.isfinite(f).all(), label
    assert (f[..., :3] >= 0).all() and (f[..., 4:] >= 0).all(), label
    w = f[..., 3]
    assert w.sum() >= samples and w.sum() <= samples * (1 + 1e-4), "%s: total weight %g for %d samples" % (
        label, w.sum(), samples)


def test_microfacet_full_resolution_same_stream(ctx, microfacet_xml):
    sid = ctx.upload(G.HostScene.load_xml(microfacet_xml))
    gfilm, st = ctx.render(sid, spp=1, batched=True)
    ofilm, paths, _ = O.Scene.load(microfacet_xml).render(0, 1, nthreads=0)
    assert st["paths"] == paths == 1024 * 1024
    # 99.97% of pixels agree to 1e-3 on this scene; the bar leaves room for rare
    # transcendental last-ulp branch flips but catches lost geometry
    same_stream_check(image(gfilm), image(ofilm), "microfacet 1024^2 x 1", min_frac=0.995)
    ctx.free_scene(sid)


def test_microfacet_statistics(ctx, microfacet_xml, tmp_path):
    # the same scene file rendered at 256 x 256 (the camera keeps its field of view)
    small = os.path.join(str(tmp_path), "microfacet_256.xml")
    with open(microfacet_xml) as f:
        txt = f.read()
    with open(small, "w") as f:
        f.write(txt.replace('name="width" value="1024"', 'name="width" value="256"')
                   .replace('name="height" value="1024"', 'name="height" value="256"'))
    assert 'value="256"' in open(small).read()
    # the OBJ files are referenced relative to the scene file's directory
    for name in os.listdir(os.path.dirname(microfacet_xml)):
        src = os.path.join(os.path.dirname(microfacet_xml), name)
        dst = os.path.join(str(tmp_path), name)
        if name != os.path.basename(microfacet_xml) and not os.path.exists(dst):
            os.symlink(src, dst)
    sid = ctx.upload(G.HostScene.load_xml(small))
    gfilm, _ = ctx.render(sid, spp=16, first_pass=100000, batched=True)   # independent seeds
    ofilm, _, _ = O.Scene.load(small).render(0, 16, nthreads=0)
    sigma_check(gfilm, ofilm, "microfacet-3sigma")
    ctx.free_scene(sid)


def test_cornell_full_size_same_stream(ctx, tmp_path):
    """The Cornell configuration as benchmarked (256^2, 16 spp, depth 8) on the oracle's
    sample streams."""
    xml = scenes.cornell(str(tmp_path), width=256, height=256, spp=16, max_depth=8)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    gfilm, st = ctx.render(sid, batched=True)
    ofilm, paths, _ = O.Scene.load(xml).render(0, 16)
    assert st["paths"] == paths == 256 * 256 * 16
    same_stream_check(image(gfilm), image(ofilm), "cornell 256^2 x 16", min_frac=0.995)
    assert np.array_equal(gfilm[..., 3], ofilm[..., 3])
    ctx.free_scene(sid)


def test_volumetric_full_size_same_stream(ctx, tmp_path):
    """The volumetric configuration at its full resolution and depth (512^2, volpath depth
    32) for 2 passes on the oracle's sample streams."""
    xml = scenes.volumetric(str(tmp_path), width=512, height=512, spp=64, max_depth=32)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    gfilm, st = ctx.render(sid, spp=2, batched=True)
    ofilm, paths, _ = O.Scene.load(xml).render(0, 2)
    assert st["paths"] == paths == 512 * 512 * 2
    same_stream_check(image(gfilm), image(ofilm), "volumetric 512^2 x 2", min_frac=0.995)
    ctx.free_scene(sid)


def test_microfacet_full_size_batched_equals_plain(ctx, microfacet_xml):
    sid = ctx.upload(G.HostScene.load_xml(microfacet_xml))
    b, sb = ctx.render(sid, spp=64, batched=True)
    p, sp = ctx.render(sid, spp=64, batched=False)
    assert sb["paths"] == sp["paths"] == 1024 * 1024 * 64
    assert np.array_equal(b[..., :4], p[..., :4])
    assert np.allclose(b[..., 4:], p[..., 4:], rtol=1e-5, atol=1e-6)
    check_film(b, 1024 * 1024 * 64, "microfacet 1024^2 x 64")
    ctx.free_scene(sid)


def test_volumetric_full_size_batched_equals_plain(ctx, tmp_path):
    xml = scenes.volumetric(str(tmp_path), width=512, height=512, spp=64, max_depth=32)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    b, sb = ctx.render(sid, batched=True)
    p, sp = ctx.render(sid, batched=False)
    assert sb["paths"] == sp["paths"] == 512 * 512 * 64
    assert np.array_equal(b[..., :4], p[..., :4])
    assert np.allclose(b[..., 4:], p[..., 4:], rtol=1e-5, atol=1e-6)
    check_film(b, 512 * 512 * 64, "volumetric 512^2 x 64")
    ctx.free_scene(sid)
