"""GPU post-processing (gnd_gpu_post) against the oracle's restatement of the reference's
post passes (tonemap.frag, bloom_*.frag, gammaCorrect.frag) and Film::savePNG's 8-bit
conversion, for every tonemap operator with and without bloom, on odd image sizes; then
a render -> post -> PNG / EXR pipeline.

Bars: tonemapped floats within 1e-4 relative (2e-4 absolute where bloom's binary16
pyramid can round the other way after a last-ulp difference of exp2 / log2 / pow);
8-bit images within one level, identical on >= 99.9% of the channels."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O

from imagefiles import read_exr, read_png

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


def hdr_image(h, w, seed):
    rng = np.random.default_rng(seed)
    img = (rng.random((h, w, 3)) ** 4 * 6).astype(np.float32)
    img[h // 3:h // 3 + 5, w // 2:w // 2 + 4] = 60.0    # a bright patch for the bloom
    img[0, :5] = 0.0
    return img


def compare(g, o, label, atol):
    gh, g8 = g
    oh, o8 = o
    assert np.allclose(gh, oh, rtol=1e-4, atol=atol), "%s: max |diff| %g" % (label, np.abs(gh - oh).max())
    d = np.abs(g8.astype(int) - o8.astype(int))
    assert d.max() <= 1 and (d == 0).mean() >= 0.999, "%s: 8-bit max %d, equal %.5f" % (label, d.max(), (d == 0).mean())


@pytest.mark.parametrize("op", range(7))
@pytest.mark.parametrize("bloom", [False, True])
def test_post_matches_oracle(ctx, op, bloom):
    img = hdr_image(61, 97, seed=op)
    kw = dict(tonemapper=op, exposure=-0.5, bloom=bloom, threshold=1.0, radius=1.0, intensity=0.04, mips=6)
    compare(ctx.post(img, **kw), O.post(img, **kw), "op %d bloom %d" % (op, bloom), atol=2e-4 if bloom else 1e-6)


def test_display_output_and_options(ctx):
    img = hdr_image(128, 256, seed=9)
    for kw in (dict(output=1), dict(output=1, tonemapper=3, bloom=True, mips=3, radius=2.0, threshold=0.5, intensity=0.2)):
        compare(ctx.post(img, **kw), O.post(img, **kw), str(kw), atol=2e-4)
    # tiny images: a pyramid of fewer levels, or none
    for h, w in ((3, 3), (5, 9), (1, 1)):
        small = hdr_image(h, w, seed=h * w)
        compare(ctx.post(small, bloom=True), O.post(small, bloom=True), "%dx%d" % (h, w), atol=2e-4)


def test_post_rejects_bad_parameters(ctx):
    img = hdr_image(8, 8, seed=1)
    for kw in (dict(tonemapper=7), dict(output=2), dict(bloom=True, mips=0), dict(bloom=True, mips=7)):
        with pytest.raises(G.GndError) as ei:
            ctx.post(img, **kw)
        assert ei.value.status == G.GND_ERR_INVALID


def test_render_post_and_files(ctx, tmp_path):
    xml = scenes.cornell(str(tmp_path), width=64, height=48, spp=8)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    film, _ = ctx.render(sid, spp=8)
    rgb = G.resolve(film)
    hdr, b8 = ctx.post(rgb, tonemapper="aces", bloom=True)
    G.write_exr(str(tmp_path / "out.exr"), hdr)
    G.write_png(str(tmp_path / "out.png"), b8)
    back, _ = read_exr(str(tmp_path / "out.exr"))
    assert np.array_equal(back, hdr)
    assert np.array_equal(read_png(str(tmp_path / "out.png")), b8)
    # the lit box is not black and ACES stays in [0, 1]
    assert b8.mean() > 10 and hdr.max() <= 1.0
    ctx.free_scene(sid)
