"""Scene uploads on a second host thread while the context is busy (gnd_gpu_scene_upload
copies, builds and validates on a stream of its own and takes the context only to
publish the scene): the render running meanwhile and the scene uploaded meanwhile both
render exactly what they render alone, with host-built and device-built mesh trees, and
uploads during serving leave the served films unchanged.

Bar: the films are bit-equal (the fixed-point film sums make renders order-independent;
the same render twice gives the same float film)."""
import threading

import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    d = tmp_path_factory.mktemp("overlap")
    # 16 x 16 displaced spheres (327,682 triangles): an upload of about 50 MB
    xml = scenes.microfacet(str(d / "m"), width=192, height=192, spp=16, max_depth=8, grid=16, seed=3)
    ctx = G.GpuContext(0)
    yield ctx, xml
    ctx.close()


def upload_in_thread(ctx, hs, n):
    out, err = [], []

    def run():
        try:
            for _ in range(n):
                out.append(ctx.upload(hs))
        except Exception as e:   # reported by the test thread
            err.append(e)

    th = threading.Thread(target=run)
    th.start()
    return th, out, err


@pytest.mark.parametrize("device_blas", [False, True])
def test_upload_during_render(setup, device_blas):
    ctx, xml = setup
    hs = G.HostScene.load_xml(xml, device_blas=device_blas)
    hs.pin(True)
    try:
        a = ctx.upload(hs)
        ref, _ = ctx.render(a, spp=16, batched=True)
        th, ids, err = upload_in_thread(ctx, hs, 3)
        during, _ = ctx.render(a, spp=16, batched=True)
        th.join()
        assert not err, err
        assert np.array_equal(during, ref), "the render during the uploads differs"
        assert len(set(ids)) == 3 and a not in ids
        for b in ids:
            info = ctx.scene_info(b)
            assert info["num_tris"] == hs.desc.num_tris and info["blas_on_device"] == int(device_blas)
            film, _ = ctx.render(b, spp=16, batched=True)
            assert np.array_equal(film, ref), "a scene uploaded during a render renders differently"
            ctx.free_scene(b)
        ctx.free_scene(a)
    finally:
        hs.pin(False)
        hs.close()


def test_upload_during_serving(setup):
    ctx, xml = setup
    hs = G.HostScene.load_xml(xml)
    a = ctx.upload(hs)
    job = dict(width=192, height=192, spp=8, max_depth=8, integrator=0)
    alone, _ = ctx.wait(ctx.submit(a, **job))
    jobs = [ctx.submit(a, first_pass=8 * k, **job) for k in range(4)]
    th, ids, err = upload_in_thread(ctx, hs, 2)
    served = [ctx.wait(j) for j in jobs]
    th.join()
    assert not err, err
    assert all(s["state"] == "done" for _, s in served)
    assert np.array_equal(served[0][0][..., :4], alone[..., :4])
    for b in ids:
        f, s = ctx.wait(ctx.submit(b, **job))
        assert s["state"] == "done" and np.array_equal(f[..., :4], alone[..., :4])
        ctx.free_scene(b)
    ctx.free_scene(a)
    hs.close()
