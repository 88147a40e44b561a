"""Motion blur on the GPU (animated.cpp, primitive.cpp:48-76, camera.h:20-25,
thinLens.cpp:80-91) against the CPU oracle: same-stream images of the Cornell box with
moving boxes and a moving area light, with camera motion, through volpath, and through a
thin lens with a rolling shutter; a toWorldEnd equal to toWorld renders bit-identically to
the static scene; batched equals plain; user ray batches (time 0) see the start state.

Bars as in the other image tests (same stream: median relative difference <= 1e-4 and
>= 99.5% of pixels within 1e-3 relative)."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O

from test_gpu_render import same_stream_check

pytestmark = pytest.mark.gpu

CASES = {
    "objects": dict(),
    "camera": dict(camera_motion=True),
    "volpath": dict(integrator="volpath_gpu"),
    "thinlens-rolling-shutter": dict(camera_motion=True,
                                     lens={"lens_radius": 0.05, "focal_distance": 3.0, "rolling_shutter": True}),
}


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_motion_same_stream(ctx, tmp_path, name):
    xml = scenes.motion(str(tmp_path), width=64, height=64, spp=4, max_depth=8, **CASES[name])
    hs = G.HostScene.load_xml(xml)
    assert hs.desc.inst_motion, "the scene has animated instances"
    sid = ctx.upload(hs)
    gfilm, st = ctx.render(sid, spp=4)
    ofilm, paths, _ = O.Scene.load(xml).render(0, 4)
    assert st["paths"] == paths
    same_stream_check(G.resolve(gfilm), G.resolve(ofilm), name, min_frac=0.995)
    ctx.free_scene(sid)


def test_equal_end_transform_is_static(ctx, tmp_path):
    """toWorldEnd equal to toWorld: no motion record, the same film sums as without it."""
    a = scenes.cornell(str(tmp_path / "a"), width=32, height=32, spp=2)
    text = open(a).read()
    start = text.index("<primitive>")
    prim_tr = text[text.index('<transform name="toWorld">', start):]
    prim_tr = prim_tr[:prim_tr.index("</transform>") + len("</transform>")]
    b = str(tmp_path / "a" / "cornell_end.xml")
    with open(b, "w") as f:
        f.write(text.replace(prim_tr, prim_tr + prim_tr.replace('name="toWorld"', 'name="toWorldEnd"'), 1))
    hb = G.HostScene.load_xml(b)
    assert not hb.desc.inst_motion
    sa, sb = ctx.upload(G.HostScene.load_xml(a)), ctx.upload(hb)
    fa, _ = ctx.render(sa, spp=2)
    fb, _ = ctx.render(sb, spp=2)
    assert np.array_equal(fa[..., :4], fb[..., :4])


def test_motion_batched_equals_plain(ctx, tmp_path):
    xml = scenes.motion(str(tmp_path), width=40, height=30, spp=6, camera_motion=True)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    a, _ = ctx.render(sid, spp=6)
    b, _ = ctx.render(sid, spp=6, batched=True)
    assert np.array_equal(a[..., :4], b[..., :4])
    ctx.free_scene(sid)


def test_user_rays_see_the_start_state(ctx, tmp_path):
    """Ray batches through gnd_gpu_trace_* carry no time: time 0, the toWorld state, so
    they hit what the oracle hits at time 0 (its rays default to time 0 as well)."""
    xml = scenes.motion(str(tmp_path), width=16, height=16, spp=1)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    rays = scenes.random_rays(1 << 15, seed=4)
    rays[:, 0:3] = rays[:, 0:3] - 0.5   # origins inside the box [-1, 1]^3
    g = ctx.trace_closest(sid, rays)
    o = O.Scene.load(xml).trace(rays)
    assert np.array_equal(g["inst"], o["inst"])
    h = g["inst"] >= 0
    assert np.allclose(g["t"][h], o["t"][h], rtol=1e-6)
    ctx.free_scene(sid)
