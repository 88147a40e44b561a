"""The exact film (gnd_gpu_render_fixed) and the work counters (gnd_gpu_counters).

Exact film: renders of disjoint pass ranges, batched or plain, add up to one render of
all the passes bit for bit (integer sums), and converted to floats they equal
gnd_gpu_render's film. Counters: the node visits and triangle tests of counted ray batches
equal the per-ray counts gnd_gpu_trace_count_dev writes, and render totals equal the sum
of the renders' own statistics."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("filt", ["box", "default"])
def test_fixed_film_sums_exactly(ctx, tmp_path, filt):
    xml = scenes.cornell(str(tmp_path), width=48, height=40, spp=6, max_depth=6, filter=filt)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    whole, wq, st = ctx.render_fixed(sid, spp=6)
    assert st["paths"] == 48 * 40 * 6
    # three calls of two passes each, alternating plain and batched, into the same buffers
    fs = np.zeros_like(whole)
    fq = np.zeros_like(wq)
    for k, batched in ((0, False), (2, True), (4, False)):
        ctx.render_fixed(sid, spp=2, first_pass=k, batched=batched, fsum=fs, fsq=fq)
    assert np.array_equal(fs, whole)
    np.testing.assert_allclose(fq, wq, rtol=1e-5, atol=1e-6)
    # the float film of gnd_gpu_render is the same sums converted
    film, _ = ctx.render(sid, spp=6)
    assert np.array_equal(G.fixed_to_film(whole, wq)[..., :4], film[..., :4])
    # every pixel has weight (the Gaussian filter spreads samples over 16 pixels)
    assert int(whole[..., 3].min()) > 0
    ctx.free_scene(sid)


def test_fixed_film_rejects_null_buffers(ctx, tmp_path):
    xml = scenes.cornell(str(tmp_path), width=8, height=8, spp=1)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    rc = G.lib().gnd_gpu_render_fixed(ctx.handle, sid, None, None, None, None)
    assert rc == G.GND_ERR_INVALID
    ctx.free_scene(sid)


def test_counters_match_trace_counts(ctx):
    import torch
    tri = scenes.random_triangles(1 << 14, seed=5)
    rays = scenes.random_rays(1 << 15, seed=5)
    sid = ctx.upload(G.HostScene.from_triangles(tri))
    ctx.counters(reset=True)
    n = rays.shape[0]
    dr = torch.from_numpy(rays).cuda()
    nodes = torch.zeros(n, dtype=torch.int32, device="cuda")
    tris = torch.zeros(n, dtype=torch.int32, device="cuda")
    ctx.trace_count_dev(sid, dr.data_ptr(), n, nodes.data_ptr(), tris.data_ptr())
    ctx.trace_closest(sid, rays[:1000])
    ctx.trace_any(sid, rays[:500])
    c = ctx.counters()
    assert c["trace_batches"] == 3
    assert c["trace_rays"] == n + 1000 + 500
    assert c["counted_rays"] == n
    assert c["counted_nodes"] == int(nodes.double().sum().item())
    assert c["counted_tris"] == int(tris.double().sum().item())
    assert c["counted_nodes"] > n   # the tree is deeper than one node
    # reset clears the sums
    c0 = ctx.counters(reset=True)
    c1 = ctx.counters()
    assert c0["trace_rays"] > 0 and c1["trace_rays"] == 0 and c1["counted_nodes"] == 0
    ctx.free_scene(sid)


def test_counters_sum_render_stats(ctx, tmp_path):
    xml = scenes.cornell(str(tmp_path), width=32, height=32, spp=3)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    ctx.counters(reset=True)
    _, a = ctx.render(sid, spp=3, profile=2)
    _, _, b = ctx.render_fixed(sid, spp=2, batched=True)
    c = ctx.counters()
    assert c["renders"] == 2
    for k in ("paths", "extend_rays", "shadow_rays", "iterations", "launches"):
        assert c[k] == a[k] + b[k], k
    # node visits and triangle tests only from the counted render
    assert c["extend_nodes"] == a["extend_nodes"] > 0 and c["extend_tris"] == a["extend_tris"]
    assert c["last"]["paths"] == b["paths"] == 32 * 32 * 2
    assert c["render_ms"] == pytest.approx(a["ms"] + b["ms"])
    # phase counters of the counted render: a warp step serves 1..32 lanes, and every
    # triangle test is a leaf step (the others enter instances or test analytic shapes)
    nw, ls, lw = a["extend_node_warp_steps"], a["extend_leaf_steps"], a["extend_leaf_warp_steps"]
    assert 0 < nw <= a["extend_nodes"] <= 32 * nw
    assert 0 < lw <= ls <= 32 * lw and ls >= a["extend_tris"]
    assert b["extend_node_warp_steps"] == b["extend_leaf_steps"] == 0
    ctx.free_scene(sid)
