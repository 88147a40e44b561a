"""Serving (gnd_gpu_serve_*): jobs that share the path pool render exactly what they
render alone and what gnd_gpu_render renders for the same arguments (same per-sample
seeds, same film sums), whatever else is running; plus cancellation, wait timeouts,
the HBM budget, a scene in use, and more jobs than the job table holds.

Bar: the fixed-point film sums (sum wL, sum w) are bit-equal; the float sum of wL^2 is
accumulated with float atomics in completion order, so it is compared within 1e-5
relative."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    d = tmp_path_factory.mktemp("serve")
    ctx = G.GpuContext(0)
    cb = ctx.upload(G.HostScene.load_xml(scenes.cornell(str(d / "c"), width=64, height=64, spp=4)))
    vol = ctx.upload(G.HostScene.load_xml(scenes.volumetric(str(d / "v"), width=48, height=48, spp=4, max_depth=16)))
    yield ctx, cb, vol, d
    ctx.close()


def same_film(a, b, label):
    assert a.shape == b.shape, label
    assert np.array_equal(a[..., :4], b[..., :4]), "%s: film sums differ on %d values" % (
        label, int((a[..., :4] != b[..., :4]).sum()))
    np.testing.assert_allclose(a[..., 4:], b[..., 4:], rtol=1e-5, atol=1e-6, err_msg=label)


def test_alone_equals_mix_equals_render(setup):
    ctx, cb, vol, _ = setup
    job = dict(width=64, height=64, spp=4, max_depth=8, integrator=0)
    ja = ctx.submit(cb, **job)
    fa, sa = ctx.wait(ja)
    assert sa["state"] == "done" and sa["samples_done"] == 64 * 64 * 4
    assert sa["submit_ms"] <= sa["admit_ms"] <= sa["done_ms"]
    fr, _ = ctx.render(cb, spp=4, max_depth=8, integrator=0)
    same_film(fa, fr, "served alone vs gnd_gpu_render")
    # the same job among others: both integrators, other sizes, depths and seeds
    ids = [ctx.submit(vol, width=48, height=48, spp=3, max_depth=12, integrator=1),
           ctx.submit(cb, width=80, height=40, spp=2, max_depth=5, integrator=0),
           ctx.submit(cb, **job),
           ctx.submit(vol, width=32, height=32, spp=5, max_depth=20, integrator=1),
           ctx.submit(cb, first_pass=4, **job)]
    out = [ctx.wait(i) for i in ids]
    assert all(s["state"] == "done" for _, s in out)
    same_film(out[2][0], fa, "in the mix vs alone")
    fv, _ = ctx.render(vol, spp=3, max_depth=12, integrator=1)
    same_film(out[0][0], fv, "volpath in the mix vs gnd_gpu_render")
    fp, _ = ctx.render(cb, spp=4, first_pass=4, max_depth=8, integrator=0)
    same_film(out[4][0], fp, "first_pass 4 in the mix vs gnd_gpu_render")
    assert out[1][0].shape == (40, 80, 7) and out[1][0][..., 3].min() > 0
    f80, _ = ctx.render(cb, spp=2, max_depth=5, integrator=0, width=80, height=40)
    same_film(out[1][0], f80, "80x40 film in the mix vs gnd_gpu_render at 80x40")


def test_more_jobs_than_the_job_table(setup):
    ctx, cb, vol, _ = setup
    ids = [ctx.submit(cb if k % 3 else vol, width=16, height=16, spp=1 + k % 4, max_depth=6, integrator=-1)
           for k in range(80)]
    for k, i in enumerate(ids):
        f, s = ctx.wait(i)
        assert s["state"] == "done" and s["samples_done"] == 16 * 16 * (1 + k % 4)
        assert np.isfinite(f).all()


def test_cancel_and_timeout(setup):
    ctx, cb, _, _ = setup
    big = ctx.submit(cb, width=256, height=256, spp=2048, max_depth=8, integrator=0)   # 134M samples
    film, st, rc = ctx.wait_any(big, timeout_ms=1)
    assert rc == G.GND_ERR_TIMEOUT and st["state"] in ("queued", "running")
    ctx.cancel_job(big)
    film, st, rc = ctx.wait_any(big)
    assert rc == G.GND_ERR_CANCELLED and st["state"] == "cancelled"
    assert st["samples_done"] < st["samples_total"]
    assert film[..., 3].sum() > 0 or st["samples_done"] == 0
    # the server keeps serving after a cancellation
    j = ctx.submit(cb, width=32, height=32, spp=2, max_depth=8, integrator=0)
    _, s = ctx.wait(j)
    assert s["state"] == "done"


def test_budget_and_scene_in_use(setup):
    ctx, _, _, d = setup
    sid = ctx.upload(G.HostScene.load_xml(scenes.cornell(str(d / "c2"), width=64, height=64, spp=4)))
    ctx.set_hbm_budget(1 << 20)
    with pytest.raises(G.GndError) as e:
        ctx.submit(sid, spp=1)
    assert e.value.status == G.GND_ERR_BUDGET
    ctx.set_hbm_budget(0)
    big = ctx.submit(sid, width=256, height=256, spp=2048, max_depth=8, integrator=0)
    with pytest.raises(G.GndError) as e:
        ctx.free_scene(sid)
    assert e.value.status == G.GND_ERR_INVALID
    ctx.cancel_job(big)
    ctx.wait_any(big)
    ctx.free_scene(sid)


@pytest.mark.parametrize("policy", ["srpt", "deadline"])
def test_small_job_overtakes_a_large_one(setup, policy):
    ctx, cb, _, _ = setup
    ctx.serve_policy(policy)
    big = ctx.submit(cb, width=256, height=256, spp=1024, max_depth=8, integrator=0)   # 67M samples
    small = ctx.submit(cb, width=16, height=16, spp=1, max_depth=8, integrator=0)
    _, ss = ctx.wait(small)
    _, sb = ctx.wait(big)
    assert ss["state"] == "done" and sb["state"] == "done"
    assert ss["done_ms"] < sb["done_ms"]
    # the small job does not wait for the big one's samples: it finishes long before
    assert (ss["done_ms"] - ss["submit_ms"]) < 0.5 * (sb["done_ms"] - sb["submit_ms"])


def test_serving_pool_size(setup):
    """The serving pool takes pool_log2 of the serving settings when no job runs; a job
    served from a 64K-slot pool (many refills per pass) renders what the default pool
    renders."""
    ctx, cb, _, _ = setup
    job = dict(width=64, height=64, spp=4, max_depth=8, integrator=0)
    ref, _ = ctx.wait(ctx.submit(cb, **job))
    try:
        ctx.serve_tune(pool_log2=16)
        small, st = ctx.wait(ctx.submit(cb, **job))
        assert st["state"] == "done"
        same_film(small, ref, "64K-slot serving pool vs the default")
    finally:
        ctx.serve_tune()
