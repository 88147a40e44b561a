"""Point, spot, directional and environment emitters on the GPU (pointlight.cpp,
spotlight.cpp, directional.cpp, environment.cpp) against the CPU oracle: same-stream
images for each light on its own and all of them together with an area light, for path
and volpath, plus an independent-seed statistical comparison of the environment-lit
scene (its importance sampling and MIS on escaping paths).

Bars as in the other image tests: same stream, median relative difference <= 1e-4 and
>= 99.5% of pixels within 1e-3 relative; statistics, <= 1% of pixel channels beyond 3
combined standard errors."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O

from test_gpu_render import same_stream_check, sigma_check

pytestmark = pytest.mark.gpu

CASES = {
    "point": dict(emitters=("point",)),
    "spot": dict(emitters=("spot",)),
    "directional": dict(emitters=("directional",)),
    "environment": dict(emitters=(), env=True),
    "all": dict(emitters=("point", "spot", "directional"), env=True, area=True),
    "volpath": dict(emitters=("point", "directional"), env=True, area=True, media=True, integrator="volpath_gpu"),
}


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_lights_same_stream(ctx, tmp_path, name):
    kw = CASES[name]
    xml = scenes.lights(str(tmp_path), width=64, height=64, spp=4, max_depth=8, **kw)
    hs = G.HostScene.load_xml(xml)
    n_em = len(kw["emitters"]) + int(kw.get("env", False)) + int(kw.get("area", False))
    assert hs.desc.num_emitters == n_em
    sid = ctx.upload(hs)
    gfilm, st = ctx.render(sid, spp=4)
    ofilm, paths, _ = O.Scene.load(xml).render(0, 4)
    assert st["paths"] == paths
    gimg = G.resolve(gfilm)
    assert gimg.mean() > 0.01, "%s: black image" % name
    same_stream_check(gimg, G.resolve(ofilm), name, min_frac=0.995)
    ctx.free_scene(sid)


def test_environment_statistics(ctx, tmp_path):
    xml = scenes.lights(str(tmp_path), width=32, height=32, spp=64, max_depth=8, emitters=("spot",), env=True)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    gfilm, _ = ctx.render(sid, spp=64, first_pass=100000)
    ofilm, _, _ = O.Scene.load(xml).render(0, 64)
    sigma_check(gfilm, ofilm, "environment-3sigma")
    ctx.free_scene(sid)


def test_batched_equals_plain_with_lights(ctx, tmp_path):
    xml = scenes.lights(str(tmp_path), width=40, height=30, spp=6, **CASES["all"])
    sid = ctx.upload(G.HostScene.load_xml(xml))
    a, _ = ctx.render(sid, spp=6)
    b, _ = ctx.render(sid, spp=6, batched=True)
    assert np.array_equal(a[..., :4], b[..., :4])
    ctx.free_scene(sid)


def test_bad_emitter_descriptions_are_refused(ctx, tmp_path):
    """An environment map whose sampling tables are missing is refused at upload."""
    import ctypes
    xml = scenes.lights(str(tmp_path), width=8, height=8, spp=1, emitters=(), env=True)
    hs = G.HostScene.load_xml(xml)
    desc = G.SceneDesc.from_address(hs._desc_ptr.value)
    saved = desc.env_dist
    desc.env_dist = None
    with pytest.raises(G.GndError) as ei:
        ctx.upload(hs)
    assert ei.value.status == G.GND_ERR_INVALID and b"environment" in G.lib().gnd_last_error()
    desc.env_dist = saved
    sid = ctx.upload(hs)
    ctx.free_scene(sid)
