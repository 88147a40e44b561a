"""Mesh trees built on the GPU at upload (gnd_gpu_scene_upload with blas_on_device):
traversal parity against the CPU oracle (whose tree is the reference's host SAH build),
the structure of the built tree (every triangle in exactly one leaf, child bounds that
contain what is below them, a consistent original -> leaf map), renders against the
host-built tree, and the scene record.

Closest hits through two different trees agree exactly except where two triangles are
at exactly the same distance (ties, counted as in the traversal tests): t is bit-equal,
and any-hit answers are identical."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O

from test_gpu_traversal import compare_closest

pytestmark = pytest.mark.gpu

K_EMPTY = 0xFFFFFFFF


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


def check_tree(nodes, tris, o2l, roots, num_tris, leaf_max=16):
    """Walks every mesh tree from its root: each triangle slot in exactly one leaf, each
    inner node reached once, every child box containing its triangles / child boxes."""
    lo_hi = nodes["lo_hi"]          # rows lox, hix, loy, hiy, loz, hiz
    child = nodes["child"]
    covered = np.zeros(num_tris, np.int32)
    seen = np.zeros(len(nodes), np.int32)
    tv = tris[:, [0, 1, 2, 4, 5, 6, 8, 9, 10]].reshape(-1, 3, 3)
    tmin, tmax = tv.min(axis=1), tv.max(axis=1)
    stack = list(roots)
    while stack:
        n = stack.pop()
        seen[n] += 1
        for k in range(4):
            c = int(child[n, k])
            if c == K_EMPTY:
                continue
            lo = lo_hi[n, [0, 2, 4], k]
            hi = lo_hi[n, [1, 3, 5], k]
            if c & 0x80000000:
                first, count = c & ((1 << 27) - 1), ((c >> 27) & 15) + 1
                assert count <= leaf_max
                covered[first:first + count] += 1
                assert (tmin[first:first + count] >= lo).all() and (tmax[first:first + count] <= hi).all()
            else:
                # the child's own children lie inside this box
                sub = child[c] != K_EMPTY
                assert (lo_hi[c, [0, 2, 4]][:, sub] >= lo[:, None]).all()
                assert (lo_hi[c, [1, 3, 5]][:, sub] <= hi[:, None]).all()
                stack.append(c)
    assert (covered == 1).all(), "slots covered %s times" % np.unique(covered)
    assert seen.max() <= 1
    # original -> leaf map: slot o2l[i] holds original triangle i (prim is mesh-local)
    assert np.array_equal(np.sort(o2l), np.arange(num_tris, dtype=np.uint32))


def device_pair(ctx, hs_dev, osc, rays, label, max_tie_frac=1e-3):
    sid = ctx.upload(hs_dev)
    try:
        info = ctx.scene_info(sid)
        assert info["blas_on_device"] == 1 and info["build_ms"] > 0.0
        gpu = ctx.trace_closest(sid, rays)
        ref = osc.trace(rays)
        st = compare_closest(gpu, ref, rays, label, max_tie_frac=max_tie_frac)
        occ_g = ctx.trace_any(sid, rays)
        occ_r, _, _ = osc.trace(rays, anyhit=True)
        assert np.array_equal(occ_g, occ_r), "%s: occlusion differs on %d rays" % (label, int((occ_g != occ_r).sum()))
        return sid, st
    except Exception:
        ctx.free_scene(sid)
        raise


def test_soup_parity_and_structure(ctx):
    tri = scenes.random_triangles(1 << 16, seed=3)
    rays = scenes.random_rays(1 << 18, seed=3)
    sid, st = device_pair(ctx, G.HostScene.from_triangles(tri, device_blas=True), O.Scene.from_triangles(tri), rays, "soup64k")
    assert st["hits"] > 10000 and st["exact_t"] == 1.0
    nodes, tris, o2l = ctx.download(sid, "nodes"), ctx.download(sid, "tris"), ctx.download(sid, "orig_to_leaf")
    check_tree(nodes, tris, o2l, roots=[1], num_tris=1 << 16)   # node 0: the top-level tree
    assert np.array_equal(tris[o2l, 3].view(np.uint32), np.arange(1 << 16, dtype=np.uint32))
    info = ctx.scene_info(sid)
    assert info["num_nodes"] == len(nodes) and info["fast_boxes"] == 1
    ctx.free_scene(sid)


def test_bounded_rays_and_coincident_triangles(ctx):
    """Equal Morton keys (many identical triangles) still split by index; their hits are
    all ties at one t."""
    rng = np.random.default_rng(9)
    tri = scenes.random_triangles(1 << 12, seed=9)
    same = np.tile(np.array([[0.4, 0.4, 0.5, 0.6, 0.4, 0.5, 0.5, 0.6, 0.5]], np.float32), (700, 1))
    tri = np.concatenate([tri.reshape(-1, 9), same])
    rays = scenes.random_rays(1 << 15, seed=9)
    rays[:, 7] = rng.uniform(0.05, 1.5, rays.shape[0]).astype(np.float32)
    rays[:, 3] = np.float32(1e-4)
    # rays that cross the stack of identical triangles
    k = 2000
    aim = np.zeros((k, 8), np.float32)
    aim[:, 0:3] = np.array([0.45, 0.45, 0.2]) + rng.uniform(-0.02, 0.02, (k, 3))
    aim[:, 4:7] = [0, 0, 1]
    aim[:, 3], aim[:, 7] = 1e-4, np.inf
    rays = np.concatenate([rays, aim])
    # most hits are on the stack, every one of them a tie
    sid, st = device_pair(ctx, G.HostScene.from_triangles(tri, device_blas=True), O.Scene.from_triangles(tri), rays,
                          "coincident", max_tie_frac=1.0)
    assert st["hits"] > 2000
    check_tree(ctx.download(sid, "nodes"), ctx.download(sid, "tris"), ctx.download(sid, "orig_to_leaf"), [1], len(tri))
    ctx.free_scene(sid)


def test_instanced_scene_render_matches_host_tree(ctx, tmp_path):
    xml = scenes.cornell(str(tmp_path), width=48, height=48, spp=4)
    a = ctx.upload(G.HostScene.load_xml(xml))
    b = ctx.upload(G.HostScene.load_xml(xml, device_blas=True))
    fa, sa = ctx.render(a, spp=4)
    fb, sb = ctx.render(b, spp=4)
    assert sa["paths"] == sb["paths"]
    # different trees: only exact-distance ties can change a path
    same = (fa[..., :4] == fb[..., :4]).all(axis=2)
    assert same.mean() >= 0.999, "%.4f of pixels identical" % same.mean()
    info = ctx.scene_info(b)
    assert info["blas_on_device"] == 1 and info["num_meshes"] > 0
    # every mesh instance got a root inside the node array, analytic shapes none
    it = ctx.download(b, "inst_trav").view(np.uint32)
    mesh = it[:, 12] == 0
    assert (it[mesh, 13] < info["num_nodes"]).all()
    ctx.free_scene(a)
    ctx.free_scene(b)


def test_many_meshes_parity(ctx, tmp_path):
    """The microfacet grid's layout, small: one mesh per sphere plus the ground, all
    built in one sort; rays across the grid against the oracle."""
    xml = scenes.microfacet(str(tmp_path), width=32, height=32, spp=1, grid=10)
    osc = O.Scene.load(xml)
    rays = scenes.random_rays(1 << 16, seed=21)
    rays[:, [0, 2]] = rays[:, [0, 2]] * 6.0 + 2.0     # origins over the 10 x 10 grid
    sid, st = device_pair(ctx, G.HostScene.load_xml(xml, device_blas=True), osc, rays, "meshes")
    assert st["hits"] > 5000
    info = ctx.scene_info(sid)
    assert info["num_meshes"] == 10 * 10 + 1
    ctx.free_scene(sid)


def test_download_checks_capacity(ctx):
    tri = scenes.random_triangles(256, seed=4)
    sid = ctx.upload(G.HostScene.from_triangles(tri, device_blas=True))
    import ctypes
    buf = np.zeros(10, np.uint32)
    st = G.lib().gnd_gpu_scene_download(ctx._h, sid, 3, buf.ctypes.data, buf.nbytes)
    assert st == G.GND_ERR_INVALID and b"too small" in G.lib().gnd_last_error()
    ctx.free_scene(sid)


def test_upload_rejects_bad_node_references(ctx):
    """A scene description whose tree points outside its arrays is refused at upload
    (checked on the device before any kernel follows a reference)."""
    import ctypes
    tri = scenes.random_triangles(512, seed=6)
    for corrupt, msg in (("inner", b"node reference out of range"), ("leaf", b"leaf range out of range")):
        hs = G.HostScene.from_triangles(tri)
        n = hs.desc.num_nodes
        child = (ctypes.c_uint32 * 4).from_address(hs.desc.nodes + (n - 1) * 128 + 96)
        if corrupt == "inner":
            child[0] = n + 5
        else:
            child[0] = 0x80000000 | (3 << 27) | (hs.desc.num_tris - 2)   # 4 triangles from the last but one
        with pytest.raises(G.GndError) as ei:
            ctx.upload(hs)
        assert ei.value.status == G.GND_ERR_INVALID and msg in G.lib().gnd_last_error()
        hs.close()
