"""Textures on the GPU (textures/perlin.h, marble.h, wood.h, cellular.h, domainWarp.h,
imageTexture.cpp) against the CPU oracle: same-stream images of the Cornell box with a
procedural or image texture on every wall and box, through path and volpath, and with a
textured area light; batched equals plain.

Bars as in the other image tests (same stream: median relative difference <= 1e-4 and
>= 99.5% of pixels within 1e-3 relative). Marble and wood go through sinf, whose last bits
differ between the device and the host; a path whose Russian roulette sits on such a
difference can diverge, which the bar allows for."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O

from test_gpu_render import same_stream_check

pytestmark = pytest.mark.gpu

CASES = {
    "path": dict(),
    "volpath": dict(integrator="volpath_gpu"),
    "textured-light": dict(emitter_texture=True),
    # every EXT feature at once: textures on moving geometry, seen through a thin lens,
    # lit by a textured area light and a point light
    "moving-lens-point": dict(emitter_texture=True, moving=True, point_light=True,
                              lens={"lens_radius": 0.04, "focal_distance": 3.5}),
    # roughness / eta / conductor eta as texture trees
    "float-textures": dict(float_textures=True),
    "float-textures-volpath": dict(float_textures=True, integrator="volpath_gpu"),
    # normal map on the back wall, bump map on the floor
    "normal-bump-maps": dict(maps=True),
    "normal-bump-maps-volpath": dict(maps=True, integrator="volpath_gpu", float_textures=True),
    # a medium-filled index box with a normal map: the medium a transmittance query enters
    # follows the perturbed normal (volPath.cpp:277)
    "index-normal-map-volpath": dict(maps=True, index_box=True, integrator="volpath_gpu"),
}


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_textures_same_stream(ctx, tmp_path, name):
    xml = scenes.textures(str(tmp_path), width=64, height=64, spp=4, max_depth=8, **CASES[name])
    hs = G.HostScene.load_xml(xml)
    assert hs.desc.num_tex_nodes > 0
    sid = ctx.upload(hs)
    gfilm, st = ctx.render(sid, spp=4)
    ofilm, paths, _ = O.Scene.load(xml).render(0, 4)
    assert st["paths"] == paths
    same_stream_check(G.resolve(gfilm), G.resolve(ofilm), name, min_frac=0.995)
    ctx.free_scene(sid)


def test_textures_batched_equals_plain(ctx, tmp_path):
    xml = scenes.textures(str(tmp_path), width=40, height=30, spp=6, emitter_texture=True)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    a, _ = ctx.render(sid, spp=6)
    b, _ = ctx.render(sid, spp=6, batched=True)
    assert np.array_equal(a[..., :4], b[..., :4])
    ctx.free_scene(sid)


def test_bad_texture_node_rejected(ctx, tmp_path):
    """A slot naming a node past the end of the tree is refused at upload."""
    xml = scenes.textures(str(tmp_path), width=16, height=16, spp=1)
    hs = G.HostScene.load_xml(xml)
    hs.desc.num_tex_nodes = 1
    with pytest.raises(G.GndError):
        ctx.upload(hs)


def test_octaves_bounded(ctx, tmp_path):
    """Perlin turbulence with more than 64 octaves is refused at upload (past ~128 octaves
    every further one only adds NaN)."""
    xml = scenes.textures(str(tmp_path), width=16, height=16, spp=1)
    text = open(xml).read().replace('<integer name="octaves" value="5"/>', '<integer name="octaves" value="65"/>', 1)
    with open(xml, "w") as f:
        f.write(text)
    hs = G.HostScene.load_xml(xml)
    with pytest.raises(G.GndError, match="octaves"):
        ctx.upload(hs)
