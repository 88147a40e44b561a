"""The host framework's texture trees (no GPU): texture objects of a scene file flattened
into gnd::TexNode records and rgba texels as the kernels read them, the texels decoded
as textureCache.h does (PNG / 255 with the sRGB curve, vertical flip, 16-bit high byte,
EXR through half precision) and checked against the oracle's image lookups, and the
errors the reference raises for bad texture descriptions."""
import ctypes
import os

import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O

TEXNODE = np.dtype([("kind", "<i4"), ("octaves", "<i4"), ("scale", "<f4"), ("strength", "<f4"),
                    ("v1", "<f4", 3), ("veinFreq", "<f4"), ("v2", "<f4", 3), ("turbScale", "<f4"),
                    ("axis", "<f4", 3), ("flags", "<i4"), ("a", "<i4"), ("b", "<i4"), ("w", "<i4"), ("h", "<i4"),
                    ("cscale", "<f4", 2), ("delta", "<f4", 2)])
assert TEXNODE.itemsize == 96


def tables(hs):
    d = hs.desc
    nodes = np.frombuffer(ctypes.string_at(d.tex_nodes, 96 * d.num_tex_nodes), TEXNODE) if d.num_tex_nodes else np.zeros(0, TEXNODE)
    texels = np.frombuffer(ctypes.string_at(d.tex_texels, 16 * d.num_tex_texels), "<f4").reshape(-1, 4) \
        if d.num_tex_texels else np.zeros((0, 4), np.float32)
    return nodes, texels


def quad_scene(tmp_path, texture_xml, extra_files=()):
    """One textured quad in front of the camera."""
    d = str(tmp_path)
    scenes.write_plane_obj(os.path.join(d, "plane.obj"))
    xml = "\n".join(["<scene>", scenes._camera((0, 0, 3), (0, 0, 0), 40, 16, 16),
                     '<sampler type="independent"/>', '<integrator type="path_gpu"/>', "<primitive>",
                     scenes._transform([("rotate", ((1, 0, 0), 90))]),
                     '<shape type="mesh"><string name="filename" value="plane.obj"/></shape>',
                     '<material type="matte">', texture_xml, "</material>", "</primitive>", "</scene>"])
    path = os.path.join(d, "quad.xml")
    with open(path, "w") as f:
        f.write(xml + "\n")
    return path


def test_textured_scene_tree():
    import tempfile
    d = tempfile.mkdtemp()
    hs = G.HostScene.load_xml(scenes.textures(d, width=16, height=16, spp=1))
    nodes, texels = tables(hs)
    kinds = sorted(nodes["kind"].tolist())
    assert kinds == [1, 2, 2, 3, 4, 5, 6, 6, 7]   # checker under the warp, two perlin, marble, wood, cellular, 2 images, warp
    warp = nodes[nodes["kind"] == 7][0]
    assert nodes[warp["a"]]["kind"] == 1 and nodes[warp["b"]]["kind"] == 2
    imgs = nodes[nodes["kind"] == 6]
    assert sorted((int(n["w"]), int(n["h"])) for n in imgs) == [(16, 12), (32, 24)]
    assert len(texels) == 32 * 24 + 16 * 12
    wood = nodes[nodes["kind"] == 4][0]
    ax = np.array([0.0, 1.0, 0.3])
    assert np.allclose(wood["axis"], ax / np.linalg.norm(ax), rtol=1e-6)
    assert wood["octaves"] == 3 and wood["veinFreq"] == np.float32(20.0) and wood["turbScale"] == np.float32(2.0)
    # default wood colours (wood.h:21-22)
    assert np.array_equal(wood["v1"], np.float32([0.6, 0.4, 0.2])) and np.array_equal(wood["v2"], np.float32([0.3, 0.15, 0.05]))


@pytest.mark.parametrize("channels", [1, 2, 3, 4])
@pytest.mark.parametrize("srgb", [False, True])
def test_png_texels_match_oracle(tmp_path, channels, srgb):
    rng = np.random.default_rng(channels + 10 * srgb)
    img = rng.integers(0, 256, (7, 5, channels)).astype(np.uint8)
    scenes.write_png(str(tmp_path / "t.png"), img)
    tex = scenes._texture("image_color", "albedo", {"filename": "t.png", "color_space": "sRGB" if srgb else "linear"})
    nodes, texels = tables(G.HostScene.load_xml(quad_scene(tmp_path, tex)))
    n = nodes[0]
    assert n["kind"] == 6 and n["w"] == 5 and n["h"] == 7 and n["b"] == channels
    # every texel centre through the oracle's closest lookup
    u, v = np.meshgrid((np.arange(5) + 0.5) / 5, (np.arange(7) + 0.5) / 7)
    uv = np.stack([u.ravel(), v.ravel()], axis=1).astype(np.float32)
    with open(tmp_path / "t.xml", "w") as f:
        f.write(tex + "\n")
    want = O.tex_eval(str(tmp_path / "t.xml"), np.zeros((35, 3), np.float32), uv=uv)
    assert np.array_equal(texels[:, :3], want)


def test_png16_and_exr_texels(tmp_path):
    img = np.random.default_rng(3).integers(0, 65536, (4, 6, 4)).astype(np.uint16)
    scenes.write_png(str(tmp_path / "a.png"), img)
    rgb = (np.random.default_rng(4).random((3, 5, 3)) * 70000 - 100).astype(np.float32)
    rgb[0, 0] = [1e-6, 65519.0, 65504.0]
    scenes.write_exr_float(str(tmp_path / "b.exr"), rgb)
    with np.errstate(over="ignore"):   # values from 65520 on become infinity, as in half precision
        half = rgb[::-1].astype(np.float16).astype(np.float32).reshape(-1, 3)
    for name, want in [("a.png", (img[::-1] >> 8).astype(np.float32).reshape(-1, 4)[:, :3] / np.float32(255)),
                       ("b.exr", half)]:
        tex = scenes._texture("image_color", "albedo", {"filename": name})
        _, texels = tables(G.HostScene.load_xml(quad_scene(tmp_path, tex)))
        assert np.array_equal(texels[:, :3], want), name


def test_shared_texture_flattened_once(tmp_path):
    """A texture object referenced by two materials becomes one node."""
    tex = scenes._texture("perlin_color", "albedo", {"scale": 0.5}).replace('name="albedo"', 'name="albedo" id="t"', 1)
    d = str(tmp_path)
    scenes.write_plane_obj(os.path.join(d, "plane.obj"))
    xml = ["<scene>", scenes._camera((0, 0, 3), (0, 0, 0), 40, 8, 8), '<sampler type="independent"/>',
           '<integrator type="path_gpu"/>']
    for k in range(2):
        xml += ["<primitive>", scenes._transform([("translate", (k, 0, 0))]),
                '<shape type="mesh"><string name="filename" value="plane.obj"/></shape>',
                '<material type="matte">', tex if k == 0 else '<ref id="t"/>', "</material>", "</primitive>"]
    xml.append("</scene>")
    with open(os.path.join(d, "s.xml"), "w") as f:
        f.write("\n".join(xml))
    nodes, _ = tables(G.HostScene.load_xml(os.path.join(d, "s.xml")))
    assert len(nodes) == 1


@pytest.mark.parametrize("body,msg", [
    (scenes._texture("image_color", "albedo", {"filename": "none.png"}), "open|load"),
    (scenes._texture("image_color", "albedo", {"filename": "x.png", "repeat_mode": "mirror"}), "repeat"),
    (scenes._texture("image_color", "albedo", {"filename": "x.png", "interpolation_mode": "cubic"}), "interpolation"),
    (scenes._texture("image_color", "albedo", {"filename": "x.png", "color_space": "aces"}), "color space"),
    (scenes._texture("domainWarp_color", "albedo", {}, [scenes._texture("perlin_color", "base", {})]), "warp"),
])
def test_texture_errors(tmp_path, body, msg):
    scenes.write_png(str(tmp_path / "x.png"), np.zeros((2, 2, 3), np.uint8))
    with pytest.raises(G.GndError, match=msg):
        G.HostScene.load_xml(quad_scene(tmp_path, body))


def test_float_texture_slots(tmp_path):
    """Float textures in roughness / eta slots become trees (Material.roughTex / etaTex =
    1 + root node); the float perlin blends with std::lerp (flag 8), the float cellular
    with Lerp; a constant float stays in the record."""
    d = str(tmp_path)
    scenes.write_plane_obj(os.path.join(d, "plane.obj"))
    xml = "\n".join(["<scene>", scenes._camera((0, 0, 3), (0, 0, 0), 40, 8, 8), '<sampler type="independent"/>',
                     '<integrator type="path_gpu"/>', "<primitive>",
                     '<shape type="mesh"><string name="filename" value="plane.obj"/></shape>',
                     '<material type="plastic">', scenes._texture("perlin_float", "roughness", {"value1": 0.1}),
                     scenes._texture("cellular_float", "eta", {"value2": 1.8}), "</material>", "</primitive>",
                     "<primitive>", '<shape type="mesh"><string name="filename" value="plane.obj"/></shape>',
                     '<material type="glass">', scenes._texture("constant_float", "roughness", {"value": 0.25}),
                     "</material>", "</primitive>", "</scene>"])
    with open(os.path.join(d, "s.xml"), "w") as f:
        f.write(xml)
    hs = G.HostScene.load_xml(os.path.join(d, "s.xml"))
    nodes, _ = tables(hs)
    mats = np.frombuffer(ctypes.string_at(hs.desc.materials, 160 * hs.desc.num_materials), "<u4").reshape(-1, 40)
    plastic = mats[mats[:, 0] == 1][0]
    glass = mats[mats[:, 0] == 3][0]
    rough, eta = nodes[plastic[3] - 1], nodes[plastic[31] - 1]
    assert rough["kind"] == 2 and rough["flags"] == 8 and rough["v1"][0] == np.float32(0.1) and rough["v2"][0] == 1.0
    assert eta["kind"] == 5 and eta["flags"] == 0 and eta["v2"][2] == np.float32(1.8)
    assert glass[3] == 0 and glass[31] == 0 and glass.view("<f4")[1] == np.float32(0.25)


def test_normal_and_bump_maps_flattened(tmp_path):
    """material.h:36-44: `normal` (image_normal) and `bump` (a float texture) children and
    bump_scale land in Material.normalTex / bumpTex / bumpScale; the normal image's node
    carries flag 16."""
    hs = G.HostScene.load_xml(scenes.textures(str(tmp_path), width=8, height=8, spp=1, maps=True))
    nodes, _ = tables(hs)
    mats = np.frombuffer(ctypes.string_at(hs.desc.materials, 160 * hs.desc.num_materials), "<u4").reshape(-1, 40)
    normal = mats[mats[:, 36] > 0]
    bump = mats[mats[:, 37] > 0]
    assert len(normal) == 1 and len(bump) == 1
    assert nodes[normal[0, 36] - 1]["kind"] == 6 and nodes[normal[0, 36] - 1]["flags"] & 16
    assert nodes[bump[0, 37] - 1]["kind"] == 2 and bump[0, 38:39].view("<f4")[0] == np.float32(0.04)
