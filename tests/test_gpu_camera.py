"""Thin-lens camera (thinLens.cpp:33-99, integrator.h:103-141) on the GPU against the CPU
oracle: same-stream images for depth of field through a disk and a polygon aperture, barrel
distortion, vignetting and chromatic aberration; the lens-less thin lens against the
pinhole camera; and batched (per-sample film records) against plain renders.

The same-stream bar is the one of the other image tests: median relative difference
<= 1e-4 and >= 99.5% of pixels within 1e-3 relative (differences come from the last ulp
of a transcendental function flipping a branch)."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O

from test_gpu_render import same_stream_check

pytestmark = pytest.mark.gpu

LENSES = {
    "dof-disk": {"lens_radius": 0.15, "focal_distance": 2.8},
    "dof-hexagon-distortion-vignetting": {"lens_radius": 0.1, "focal_distance": 3.2, "blades": 6, "k1": 0.15,
                                          "vignetting": True},
    "chromatic-aberration": {"lens_radius": 0.08, "focal_distance": 3.0, "ca_axial": 0.05, "ca_lateral": 0.02,
                             "vignetting": True},
}


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(LENSES))
def test_thin_lens_same_stream(ctx, tmp_path, name):
    xml = scenes.cornell(str(tmp_path), width=64, height=64, spp=4, lens=LENSES[name])
    sid = ctx.upload(G.HostScene.load_xml(xml))
    gfilm, st = ctx.render(sid, spp=4)
    ofilm, paths, _ = O.Scene.load(xml).render(0, 4)
    assert st["paths"] == paths == 64 * 64 * 4
    same_stream_check(G.resolve(gfilm), G.resolve(ofilm), name, min_frac=0.995)


def test_lensless_thin_lens_equals_pinhole(ctx, tmp_path):
    """lens_radius 0 without distortion or aberration: the same rays as the pinhole
    camera, so the fixed-point film sums are bit-identical."""
    a = ctx.upload(G.HostScene.load_xml(scenes.cornell(str(tmp_path / "a"), width=40, height=40, spp=3)))
    b = ctx.upload(G.HostScene.load_xml(scenes.cornell(str(tmp_path / "b"), width=40, height=40, spp=3,
                                                       lens={"focal_distance": 5.0})))
    fa, _ = ctx.render(a, spp=3)
    fb, _ = ctx.render(b, spp=3)
    assert np.array_equal(fa[..., :4], fb[..., :4])


def test_thin_lens_batched_equals_plain(ctx, tmp_path):
    xml = scenes.cornell(str(tmp_path), width=40, height=30, spp=6, lens=LENSES["chromatic-aberration"])
    sid = ctx.upload(G.HostScene.load_xml(xml))
    a, sa = ctx.render(sid, spp=6)
    b, sb = ctx.render(sid, spp=6, batched=True)
    assert sa["paths"] == sb["paths"] == 40 * 30 * 6
    assert np.array_equal(a[..., :4], b[..., :4])
    assert np.allclose(a[..., 4:], b[..., 4:], rtol=1e-5, atol=1e-6)
