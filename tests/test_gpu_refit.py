"""BVH refit on the GPU (gnd_gpu_scene_refit_mesh): a resident mesh takes new positions
and keeps its tree topology. Closest hits after a refit equal those of a scene built from
the new positions (same triangle, same t; only exact ties between triangles may resolve
differently), a refitted Cornell box with taller boxes renders like the oracle's scene
file with the deformed mesh (same-stream bar of the other image tests), a second refit
back to the old positions restores the old hits, and the refusals hold."""
import os

import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O

from test_gpu_render import same_stream_check

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = G.GpuContext(0)
    yield c
    c.close()


def _hits_agree(a, b, max_ties=1e-4):
    same = (a["inst"] == b["inst"]) & (a["prim"] == b["prim"])
    assert np.mean(~same) <= max_ties, "hits differ for %d rays" % int((~same).sum())
    assert np.array_equal(a["t"][same], b["t"][same])
    # where the triangle differs, the distance is the same (a tie)
    assert np.allclose(a["t"][~same], b["t"][~same], rtol=1e-6)


def test_refit_matches_rebuild(ctx):
    t0 = scenes.random_triangles(1 << 16, seed=11).reshape(-1, 9)
    rng = np.random.default_rng(12)
    t1 = t0 + rng.normal(0, 0.02, t0.shape).astype(np.float32)
    t1[:, 1::3] *= 1.5   # stretch every vertex in y: boxes grow beyond the old tree's
    rays = scenes.random_rays(1 << 18, seed=13)
    sid = ctx.upload(G.HostScene.from_triangles(t0))
    before = ctx.trace_closest(sid, rays)
    ms = ctx.refit_mesh(sid, 0, t1)
    assert ms > 0.0
    fresh = ctx.upload(G.HostScene.from_triangles(t1))
    _hits_agree(ctx.trace_closest(sid, rays), ctx.trace_closest(fresh, rays))
    assert np.array_equal(ctx.trace_any(sid, rays), ctx.trace_any(fresh, rays))
    # back to the old positions: the old tree's boxes again, the old hits
    ctx.refit_mesh(sid, 0, t0)
    again = ctx.trace_closest(sid, rays)
    assert np.array_equal(again["inst"], before["inst"]) and np.array_equal(again["prim"], before["prim"])
    assert np.array_equal(again["t"], before["t"])
    ctx.free_scene(sid)
    ctx.free_scene(fresh)


def test_refit_device_built_tree(ctx):
    t0 = scenes.random_triangles(1 << 15, seed=21).reshape(-1, 9)
    t1 = t0 * np.float32(1.25) + np.float32(0.1)
    rays = scenes.random_rays(1 << 17, seed=22)
    sid = ctx.upload(G.HostScene.from_triangles(t0, device_blas=True))
    ctx.refit_mesh(sid, 0, t1)
    fresh = ctx.upload(G.HostScene.from_triangles(t1))
    _hits_agree(ctx.trace_closest(sid, rays), ctx.trace_closest(fresh, rays))
    ctx.free_scene(sid)
    ctx.free_scene(fresh)


def _cube_triangles(path):
    """Corner positions of an OBJ's triangles in face order (9 floats each)."""
    v, tris = [], []
    for line in open(path):
        p = line.split()
        if p and p[0] == "v":
            v.append([float(x) for x in p[1:4]])
        elif p and p[0] == "f":
            tris.append([v[int(c.split("/")[0]) - 1] for c in p[1:4]])
    return np.array(tris, np.float32).reshape(-1, 9)


def test_refit_cornell_renders_like_oracle(ctx, tmp_path):
    xml = scenes.cornell(str(tmp_path), width=64, height=64, spp=4)
    cube = os.path.join(str(tmp_path), "cube.obj")
    # the deformed cube: 1.35 times taller, shifted in x, written as a second OBJ file
    lines = []
    for line in open(cube):
        p = line.split()
        if p and p[0] == "v":
            x, y, z = (float(a) for a in p[1:4])
            line = "v %r %r %r\n" % (float(np.float32(x + 0.1)), float(np.float32(y * 1.35)), z)
        lines.append(line)
    with open(os.path.join(str(tmp_path), "cube2.obj"), "w") as f:
        f.writelines(lines)
    xml2 = os.path.join(str(tmp_path), "cornell2.xml")
    with open(xml2, "w") as f:
        f.write(open(xml).read().replace('"cube.obj"', '"cube2.obj"'))
    new = _cube_triangles(os.path.join(str(tmp_path), "cube2.obj"))
    sid = ctx.upload(G.HostScene.load_xml(xml))
    meshes = ctx.scene_info(sid)["num_meshes"]
    done = False
    for m in range(meshes):   # the cube is the mesh with 12 triangles
        try:
            ctx.refit_mesh(sid, m, new)
            done = True
        except G.GndError as e:
            assert "triangles" in str(e) or "area light" in str(e)
    assert done
    gfilm, st = ctx.render(sid, spp=4)
    ofilm, paths, _ = O.Scene.load(xml2).render(0, 4)
    assert st["paths"] == paths
    same_stream_check(G.resolve(gfilm), G.resolve(ofilm), "refit-cornell", min_frac=0.995)
    fresh = ctx.upload(G.HostScene.load_xml(xml2))
    ffilm, _ = ctx.render(fresh, spp=4)
    same_stream_check(G.resolve(gfilm), G.resolve(ffilm), "refit-vs-rebuild", min_frac=0.995)
    ctx.free_scene(sid)
    ctx.free_scene(fresh)


def test_refit_refusals(ctx, tmp_path):
    t0 = scenes.random_triangles(1024, seed=3).reshape(-1, 9)
    sid = ctx.upload(G.HostScene.from_triangles(t0))
    with pytest.raises(G.GndError, match="triangles"):
        ctx.refit_mesh(sid, 0, t0[:-1])
    with pytest.raises(G.GndError, match="out of range"):
        ctx.refit_mesh(sid, 1, t0)
    bad = t0.copy()
    bad[5, 4] = np.nan
    with pytest.raises(G.GndError, match="finite"):
        ctx.refit_mesh(sid, 0, bad)
    ctx.free_scene(sid)
    # the light's plane mesh of the Cornell box carries an area light
    xml = scenes.cornell(str(tmp_path / "c"), width=16, height=16, spp=1)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    plane = np.array([[-1, 0, -1, 1, 0, -1, 1, 0, 1], [-1, 0, -1, 1, 0, 1, -1, 0, 1]], np.float32)
    msgs = []
    for m in range(ctx.scene_info(sid)["num_meshes"]):
        try:
            ctx.refit_mesh(sid, m, plane)
        except G.GndError as e:
            msgs.append(str(e))
    assert any("area light" in s for s in msgs)
    ctx.free_scene(sid)
    # moving instances
    mx = scenes.motion(str(tmp_path / "m"), width=16, height=16, spp=1)
    sid = ctx.upload(G.HostScene.load_xml(mx))
    with pytest.raises(G.GndError, match="moving"):
        ctx.refit_mesh(sid, 0, plane)
    ctx.free_scene(sid)


def test_refit_refused_while_jobs_use_the_scene(ctx, tmp_path):
    """A served job that names the scene (queued or running) blocks a refit, which would
    change the geometry between the job's rounds; once the job is done the refit runs."""
    xml = scenes.cornell(str(tmp_path / "c"), width=64, height=64, spp=4)
    hs = G.HostScene.load_xml(xml)
    sid = ctx.upload(hs)
    cube = _cube_triangles(os.path.join(str(tmp_path / "c"), "cube.obj"))
    box = None   # the cube mesh (12 triangles, no area light)
    for m in range(ctx.scene_info(sid)["num_meshes"]):
        try:
            ctx.refit_mesh(sid, m, cube)
            box = m
            break
        except G.GndError:
            continue
    assert box is not None
    big = ctx.submit(sid, width=256, height=256, spp=2048, max_depth=8, integrator=0)
    with pytest.raises(G.GndError, match="jobs") as e:
        ctx.refit_mesh(sid, box, cube)
    assert e.value.status == G.GND_ERR_INVALID
    ctx.cancel_job(big)
    ctx.wait_any(big)
    ctx.refit_mesh(sid, box, cube)
    ctx.free_scene(sid)
