"""GPU traversal parity: gnd_gpu_trace_closest / gnd_gpu_trace_any against the CPU
oracle's restatement of the reference BVH4 traversal (bvhTraversal.h:19-98,
mesh.cpp:231-326, bvh.cpp:38-66) on identical ray batches.

Bar: the same hit primitive (instance + triangle), t within 1e-6 relative (the kernels
reproduce the reference's separately rounded arithmetic, so t is expected bit-equal),
same occlusion answer. Shared-edge ties (two primitives at exactly equal t) may resolve
differently because the GPU visits children front to back; they are counted and listed,
never treated as failures, and must stay rare."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

T_REL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


def compare_closest(gpu, ref, rays, label, max_tie_frac=1e-3):
    g_hit = gpu["inst"] >= 0
    r_hit = ref["inst"] >= 0
    assert np.array_equal(g_hit, r_hit), "%s: hit/miss differs on %d rays" % (label, int((g_hit != r_hit).sum()))
    h = g_hit
    same = (gpu["inst"][h] == ref["inst"][h]) & (gpu["prim"][h] == ref["prim"][h])
    tg, tr = gpu["t"][h], ref["t"][h]
    rel = np.abs(tg - tr) / np.maximum(np.abs(tr), 1e-30)
    # a differing primitive at the same t is a tie; anything else is a failure
    tie = ~same & (tg == tr)
    bad = ~same & ~tie
    assert not bad.any(), "%s: %d rays hit a different primitive at a different t, e.g. %s" % (
        label, int(bad.sum()), list(zip(gpu["inst"][h][bad][:5], gpu["prim"][h][bad][:5], ref["inst"][h][bad][:5], ref["prim"][h][bad][:5])))
    assert rel.max(initial=0) <= T_REL, "%s: max relative t error %g" % (label, rel.max())
    tie_frac = float(tie.mean()) if tie.size else 0.0
    assert tie_frac <= max_tie_frac, "%s: %d ties" % (label, int(tie.sum()))
    # barycentrics of matching hits come out of the same arithmetic
    assert np.allclose(gpu["u"][h][same], ref["u"][h][same], atol=1e-6)
    assert np.allclose(gpu["v"][h][same], ref["v"][h][same], atol=1e-6)
    return dict(hits=int(h.sum()), ties=int(tie.sum()), exact_t=float((tg == tr).mean()) if h.any() else 1.0)


def run_pair(ctx, hs, osc, rays, label):
    sid = ctx.upload(hs)
    try:
        gpu = ctx.trace_closest(sid, rays)
        ref = osc.trace(rays)
        stats = compare_closest(gpu, ref, rays, label)
        occ_g = ctx.trace_any(sid, rays)
        occ_r, _, _ = osc.trace(rays, anyhit=True)
        assert np.array_equal(occ_g, occ_r), "%s: occlusion differs on %d rays" % (label, int((occ_g != occ_r).sum()))
        # any-hit agrees with "a closest hit exists" for unbounded rays
        unb = np.isinf(rays[:, 7])
        assert np.array_equal(occ_g[unb], gpu["inst"][unb] >= 0)
        return stats
    finally:
        ctx.free_scene(sid)


def test_soup_parity(ctx):
    tri = scenes.random_triangles(1 << 16, seed=3)
    rays = scenes.random_rays(1 << 18, seed=3)
    st = run_pair(ctx, G.HostScene.from_triangles(tri), O.Scene.from_triangles(tri), rays, "soup64k")
    assert st["hits"] > 10000 and st["exact_t"] == 1.0


def test_soup_bounded_rays(ctx):
    tri = scenes.random_triangles(1 << 14, seed=5)
    rays = scenes.random_rays(1 << 16, seed=5)
    rays[:, 7] = np.random.default_rng(5).uniform(0.01, 0.5, rays.shape[0]).astype(np.float32)
    rays[:, 3] = np.float32(1e-4)
    run_pair(ctx, G.HostScene.from_triangles(tri), O.Scene.from_triangles(tri), rays, "soup-bounded")


def test_empty_and_degenerate_batches(ctx):
    tri = scenes.random_triangles(64, seed=1)
    hs = G.HostScene.from_triangles(tri)
    sid = ctx.upload(hs)
    assert ctx.trace_closest(sid, np.zeros((0, 8), np.float32)).shape == (0,)
    # rays along axes (zero direction components -> infinite inverse directions)
    r = np.array([[0.5, 0.5, -1, 1e-4, 0, 0, 1, np.inf], [0.5, -1, 0.5, 1e-4, 0, 1, 0, np.inf],
                  [-1, 0.5, 0.5, 1e-4, 1, 0, 0, np.inf], [5, 5, 5, 1e-4, 1, 1, 1, np.inf]], np.float32)
    g = ctx.trace_closest(sid, r)
    ref = O.Scene.from_triangles(tri).trace(r)
    assert np.array_equal(g["inst"], ref["inst"]) and np.array_equal(g["prim"], ref["prim"])
    ctx.free_scene(sid)


def _scene_rays(osc, w, h, n_random, seed, lo=-1.0, hi=1.0):
    px, py = np.meshgrid(np.arange(w), np.arange(h))
    cam = osc.camera_rays(0, px.ravel(), py.ravel())
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n_random, 3))
    d = rng.normal(size=(n_random, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rnd = np.concatenate([o, np.full((n_random, 1), 1e-4), d, np.full((n_random, 1), np.inf)], axis=1).astype(np.float32)
    return np.concatenate([cam, rnd]).astype(np.float32)


def test_cornell_parity(ctx, tmp_path):
    xml = scenes.cornell(str(tmp_path), width=64, height=64)
    osc = O.Scene.load(xml)
    rays = _scene_rays(osc, 64, 64, 100000, 11, -0.99, 0.99)
    run_pair(ctx, G.HostScene.load_xml(xml), osc, rays, "cornell")


def test_volumetric_scene_parity(ctx, tmp_path):
    # analytic sphere, index-material cube mesh, rotated / scaled instances
    xml = scenes.volumetric(str(tmp_path), width=48, height=48)
    osc = O.Scene.load(xml)
    rays = _scene_rays(osc, 48, 48, 100000, 12, -0.99, 0.99)
    run_pair(ctx, G.HostScene.load_xml(xml), osc, rays, "volumetric")


def test_analytic_shapes_parity(ctx, tmp_path):
    (tmp_path / "a.xml").write_text("""<scene>
<camera type="perspective"><transform name="toWorld"><lookat origin="0,0,6" target="0,0,0" up="0,1,0"/></transform></camera>
<sampler type="independent"/><integrator type="path_gpu"/>
<primitive><transform name="toWorld"><scale value="1.5"/><rotate axis="1 1 0" angle="30"/><translate x="-1" y="0" z="0"/></transform>
<shape type="sphere"><float name="radius" value="0.7"/></shape></primitive>
<primitive><transform name="toWorld"><rotate axis="0 1 1" angle="40"/><translate x="1.2" y="0.3" z="-0.5"/></transform>
<shape type="cube"><vector name="extents" value="0.5, 0.8, 0.3"/></shape>
<emitter type="area"><color name="radiance" value="1 1 1"/></emitter></primitive>
</scene>""")
    xml = str(tmp_path / "a.xml")
    osc = O.Scene.load(xml)
    rays = _scene_rays(osc, 32, 32, 200000, 13, -3, 3)
    run_pair(ctx, G.HostScene.load_xml(xml), osc, rays, "analytic")


def test_translated_instances_parity(ctx, tmp_path):
    """Mesh, sphere and cube instances under pure translations (one with a zero
    component) beside rotated and scaled ones, traced with rays whose origins lie on an
    integer grid (many zero components, so the transformed origins carry signed zeros) and
    rays along the axes (infinite inverse directions): the oracle's hits."""
    scenes.write_cube_obj(str(tmp_path / "cube.obj"))
    scenes.write_plane_obj(str(tmp_path / "plane.obj"))

    def prim(shape, xf):
        return "<primitive><transform name=\"toWorld\">%s</transform>%s</primitive>" % (xf, shape)

    mesh = "<shape type=\"mesh\"><string name=\"filename\" value=\"%s\"/></shape>"
    parts = [prim(mesh % "cube.obj", '<translate x="1.25" y="-0.75" z="0.5"/>'),
             prim(mesh % "cube.obj", '<translate x="-1.5" y="0" z="-0.25"/>'),
             prim(mesh % "cube.obj", '<translate x="-0.375" y="-0.625" z="-1.75"/>'),
             prim(mesh % "plane.obj", '<rotate axis="1 0 0" angle="90"/><translate x="0.125" y="-1.5" z="0.375"/>'),
             prim(mesh % "cube.obj", '<rotate axis="0 1 1" angle="35"/><scale value="0.35"/><translate x="0.2" y="1.1" z="-1.3"/>'),
             prim('<shape type="sphere"><float name="radius" value="0.45"/></shape>', '<translate x="-0.6" y="0.7" z="1.2"/>'),
             prim('<shape type="cube"><vector name="extents" value="0.3, 0.2, 0.4"/></shape>'
                  '<emitter type="area"><color name="radiance" value="1 1 1"/></emitter>', '<translate x="0.9" y="0.8" z="-0.3"/>')]
    (tmp_path / "t.xml").write_text(
        '<scene><camera type="perspective"><transform name="toWorld"><lookat origin="0.3,0.2,5" target="0,0,0" up="0,1,0"/>'
        '</transform></camera><sampler type="independent"/><integrator type="path_gpu"/>' + "".join(parts) + '</scene>')
    xml = str(tmp_path / "t.xml")
    osc = O.Scene.load(xml)
    rays = _scene_rays(osc, 32, 32, 150000, 14, -2.5, 2.5)
    rng = np.random.default_rng(15)
    n = rays.shape[0]
    # origins on a coarse grid: many components exactly zero
    grid = rng.random(n) < 0.25
    rays[grid, :3] = rng.integers(-2, 3, (int(grid.sum()), 3)).astype(np.float32)
    # some axis-aligned directions (zero components: infinite inverse direction)
    axis = rng.random(n) < 0.05
    k = rng.integers(0, 3, int(axis.sum()))
    d = np.zeros((int(axis.sum()), 3), np.float32)
    d[np.arange(len(k)), k] = rng.choice([-1.0, 1.0], len(k))
    rays[axis, 4:7] = d
    st = run_pair(ctx, G.HostScene.load_xml(xml), osc, rays, "translated")
    assert st["hits"] > 20000


def test_full_size_traversal_parity(ctx):
    """The traversal micro-benchmark's full scene (2^20 triangles); a 2^21-ray sample of
    its 2^24 rays is compared with the oracle, and any-hit is checked against closest-hit
    on the whole 2^24 batch (a size-independent property)."""
    tri = scenes.random_triangles(1 << 20, seed=1)
    rays = scenes.random_rays(1 << 24, seed=1)
    hs = G.HostScene.from_triangles(tri)
    sid = ctx.upload(hs)
    try:
        sample = rays[:: 8]
        gpu = ctx.trace_closest(sid, sample)
        ref = O.Scene.from_triangles(tri).trace(sample)
        st = compare_closest(gpu, ref, sample, "full-size")
        assert st["hits"] > 100000
        allh = ctx.trace_closest(sid, rays)
        occ = ctx.trace_any(sid, rays)
        assert np.array_equal(occ, allh["inst"] >= 0)
        assert np.array_equal(allh[::8], gpu)
    finally:
        ctx.free_scene(sid)


def test_key_ordered_batches(ctx):
    """ray_sort bit 2 and trace_leaf_batch: a batch traversed in ray-key order, or with the
    warps' node phases cut short at any leaf count, gives every ray the same result in its
    own slot (closest hit, occlusion, node and triangle counts) as input order with full
    node phases, and matches the oracle; each ray's traversal does not depend on the other
    rays."""
    torch = pytest.importorskip("torch")
    tri = scenes.random_triangles(1 << 18, seed=4)
    rays = scenes.random_rays(1 << 20, seed=4)
    hs = G.HostScene.from_triangles(tri)
    sid = ctx.upload(hs)
    try:
        out = {}
        for rs, lb, tb in ((0, 32, 8), (4, 12, 8), (0, 1, 9), (4, 7, 10), (0, 12, 9)):
            ctx.set_tune(sid, ray_sort=rs, trace_leaf_batch=lb, trace_blocks=tb)
            closest = ctx.trace_closest(sid, rays)
            occ = ctx.trace_any(sid, rays)
            dr = torch.from_numpy(rays).cuda()
            nodes = torch.zeros(rays.shape[0], dtype=torch.int32, device="cuda")
            tris = torch.zeros(rays.shape[0], dtype=torch.int32, device="cuda")
            ctx.trace_count_dev(sid, dr.data_ptr(), rays.shape[0], nodes.data_ptr(), tris.data_ptr())
            torch.cuda.synchronize()
            out[(rs, lb, tb)] = (closest, occ, nodes.cpu().numpy(), tris.cpu().numpy())
        a = out[(0, 32, 8)]
        for key, b in out.items():
            assert a[0].tobytes() == b[0].tobytes(), key
            assert np.array_equal(a[1], b[1]), key
            assert np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3]), key
        b = out[(4, 12, 8)]
        sample = rays[::16]
        ref = O.Scene.from_triangles(tri).trace(sample)
        compare_closest(b[0][::16], ref, sample, "key-ordered")
    finally:
        ctx.set_tune(sid, ray_sort=0, trace_leaf_batch=12, trace_blocks=8)
        ctx.free_scene(sid)


def test_device_pointer_variant_matches_host(ctx):
    torch = pytest.importorskip("torch")
    tri = scenes.random_triangles(1 << 12, seed=9)
    rays = scenes.random_rays(1 << 14, seed=9)
    hs = G.HostScene.from_triangles(tri)
    sid = ctx.upload(hs)
    host = ctx.trace_closest(sid, rays)
    dr = torch.from_numpy(rays).cuda()
    dh = torch.zeros((rays.shape[0], 5), dtype=torch.int32, device="cuda")
    ctx.trace_closest_dev(sid, dr.data_ptr(), rays.shape[0], dh.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    dev = dh.cpu().numpy().view(G.HIT_DTYPE).reshape(-1)
    assert np.array_equal(dev, host)
    nodes = torch.zeros(rays.shape[0], dtype=torch.int32, device="cuda")
    tris = torch.zeros(rays.shape[0], dtype=torch.int32, device="cuda")
    ctx.trace_count_dev(sid, dr.data_ptr(), rays.shape[0], nodes.data_ptr(), tris.data_ptr(),
                        torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(nodes.sum()) > rays.shape[0] and int(tris.sum()) > 0
    ctx.free_scene(sid)


def test_upload_rejects_corrupted_node_reference(ctx):
    import ctypes
    tri = scenes.random_triangles(256, seed=2)
    hs = G.HostScene.from_triangles(tri)
    # point a child reference of the root past the node array (host copy only)
    addr = hs.desc.nodes + 96
    old = ctypes.c_uint32.from_address(addr).value
    ctypes.c_uint32.from_address(addr).value = 0x7FFFFFF0
    try:
        with pytest.raises(G.GndError) as ei:
            ctx.upload(hs)
        assert ei.value.status == 1
    finally:
        ctypes.c_uint32.from_address(addr).value = old
