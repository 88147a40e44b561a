"""CPU-side checks of the native library: it loads, exports every symbol the public
header declares, the host scene framework builds valid BVH4 layouts, and GPU entry
points fail loudly (no CPU fallback) when no CUDA device is present."""
import os
import re

import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMPTY = 0xFFFFFFFF
LEAF = 0x80000000


def header_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            text = open(os.path.join(ROOT, "include", f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(gnd_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = G.lib()
    names = header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in G.lib().gnd_version()


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="a CUDA device is present")
def test_gpu_context_fails_loudly_without_device():
    with pytest.raises(G.GpuUnavailable):
        G.GpuContext(0)


def _check_bvh(hs, expect_tris):
    """Every triangle slot is referenced by exactly one leaf and every child box contains
    what it references."""
    nodes = hs.nodes()
    tris = hs.tris().reshape(-1, 3, 4)[:, :, :3]
    tl = hs.tlas_list()
    inst = hs.inst_trav()
    seen = np.zeros(len(tris), np.int32)
    roots = [int(row[13]) for row in inst if int(row[12]) == 0 and int(row[13]) != EMPTY]

    def visit(n, lo, hi, top):
        node = nodes[n]
        box = node["lo_hi"]  # lox, hix, loy, hiy, loz, hiz
        for k in range(4):
            c = int(node["child"][k])
            if c == EMPTY:
                continue
            clo = np.array([box[0][k], box[2][k], box[4][k]])
            chi = np.array([box[1][k], box[3][k], box[5][k]])
            if lo is not None:
                assert np.all(clo >= lo - 1e-6) and np.all(chi <= hi + 1e-6)
            if c & LEAF:
                first, count = c & ((1 << 27) - 1), ((c >> 27) & 15) + 1
                if top:
                    assert first + count <= len(tl)
                else:
                    for s in range(first, first + count):
                        seen[s] += 1
                        assert np.all(tris[s] >= clo - 1e-6) and np.all(tris[s] <= chi + 1e-6)
            else:
                visit(c, clo, chi, top)

    visit(int(hs.desc.tlas_root), None, None, True)
    for r in set(roots):
        visit(r, None, None, False)
    assert seen.sum() == expect_tris and np.all(seen == 1)
    assert sorted(tl.tolist()) == list(range(hs.desc.num_instances))


def test_host_bvh_soup_valid():
    tri = scenes.random_triangles(5000, seed=7)
    hs = G.HostScene.from_triangles(tri)
    assert hs.desc.num_tris == 5000 and hs.desc.num_instances == 1
    _check_bvh(hs, 5000)


def test_host_bvh_coincident_centroids_split_large_leaves():
    # 100 copies of one triangle: the builder makes one 100-primitive leaf (equal
    # centroids, bvhBuilder.cpp:94-96); the layout splits it into <=16-triangle leaves.
    t = np.tile(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)[None], (100, 1, 1))
    hs = G.HostScene.from_triangles(t)
    _check_bvh(hs, 100)


def test_host_cornell_scene(tmp_path):
    hs = G.HostScene.load_xml(scenes.cornell(str(tmp_path)))
    d = hs.desc
    assert (d.width, d.height, d.spp, d.max_depth, d.integrator, d.filter) == (256, 256, 16, 8, 0, 0)
    assert d.num_instances == 8 and d.num_emitters == 1 and d.num_tris == 2 + 12
    _check_bvh(hs, 14)


def test_host_volumetric_scene(tmp_path):
    hs = G.HostScene.load_xml(scenes.volumetric(str(tmp_path), width=64, height=48))
    d = hs.desc
    assert (d.width, d.height, d.integrator) == (64, 48, 1)
    assert d.num_instances == 10 and d.num_media == 3


@pytest.mark.parametrize("xml,needle", [
    ("<scene><bogus/></scene>", "not registered"),
    ("<scene><primitive></scene>", "closes"),
    ("<scene><primitive><shape type=\"mesh\"><string name=\"filename\" value=\"nope.obj\"/></shape></primitive></scene>", "Failed to load OBJ"),
    ("<scene><primitive/></scene>", "without a Shape"),
    ("<scene><shape type=\"sphere\"/></scene>", "cannot add"),
])
def test_host_errors_are_reported(tmp_path, xml, needle):
    p = tmp_path / "s.xml"
    p.write_text(xml)
    with pytest.raises(G.GndError) as ei:
        G.HostScene.load_xml(str(p))
    assert ei.value.status == 6 and needle in str(ei.value)


def test_obj_loader_polygons_and_negative_indices(tmp_path):
    (tmp_path / "q.obj").write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf -4 -3 -2 -1\n")
    (tmp_path / "s.xml").write_text(
        '<scene><camera type="perspective"/><sampler type="independent"/><integrator type="path_gpu"/>'
        '<primitive><shape type="mesh"><string name="filename" value="q.obj"/></shape>'
        '<emitter type="area"><color name="radiance" value="1 1 1"/></emitter></primitive></scene>')
    hs = G.HostScene.load_xml(str(tmp_path / "s.xml"))
    assert hs.desc.num_tris == 2
    _check_bvh(hs, 2)


def _mesh_scene(tmp_path, names):
    prims = "".join(
        f'<primitive><shape type="mesh"><string name="filename" value="{n}"/></shape>'
        '<emitter type="area"><color name="radiance" value="1 1 1"/></emitter></primitive>' for n in names)
    (tmp_path / "s.xml").write_text(
        '<scene><camera type="perspective"/><sampler type="independent"/><integrator type="path_gpu"/>'
        + prims + '</scene>')
    return str(tmp_path / "s.xml")


def test_obj_loader_number_forms(tmp_path):
    """Coordinates are strtod's values rounded to float in every written form (a sign,
    hexadecimal, values below the float range, more digits than a double holds, tabs,
    CRLF line ends, a comment after a face, no newline at the end)."""
    vs = [("+1.25", "\t-0.5", "1e-50"), ("1e-40", "0x1.8p1", "2.9999999999999999"),
          ("1.000000000000000000000001", "-0", "  7"), ("4.9e-324", "1.17549435e-38", "0.1")]
    text = "".join(f"v {a} {b} {c}\r\n" for a, b, c in vs) + "f +1 2 3 #tri\r\nf\t-1 -2 -3"
    (tmp_path / "n.obj").write_text(text, newline="")

    def val(s):
        s = s.strip()
        return np.float32(float.fromhex(s) if "0x" in s else float(s))

    want = np.array([[val(x) for x in v] for v in vs], np.float32)
    hs = G.HostScene.load_xml(_mesh_scene(tmp_path, ["n.obj"]), device_blas=True)
    got = hs.tris().reshape(-1, 3, 4)[:, :, :3]
    assert got.tobytes() == want[[0, 1, 2, 3, 2, 1]].reshape(2, 3, 3).tobytes()


@pytest.mark.parametrize("device_blas", [False, True])
def test_flatten_many_meshes(tmp_path, device_blas):
    """Meshes are concatenated in first-use order, each triangle at its mesh's base plus its
    leaf position; one mesh spans more than one 65,536-triangle piece of the flattening."""
    rng = np.random.default_rng(5)
    sizes = [3, 70001, 1, 500]
    meshes = []
    for k, n in enumerate(sizes):
        p = (rng.random((n, 3, 3)) + k).astype(np.float32)
        meshes.append(p)
        lines = [f"v {x!r} {y!r} {z!r}" for x, y, z in p.reshape(-1, 3).astype(np.float64).tolist()]
        lines += [f"f {3 * t + 1} {3 * t + 2} {3 * t + 3}" for t in range(n)]
        (tmp_path / f"m{k}.obj").write_text("\n".join(lines) + "\n")
    hs = G.HostScene.load_xml(_mesh_scene(tmp_path, [f"m{k}.obj" for k in range(len(sizes))]),
                              device_blas=device_blas)
    tris = hs.tris().reshape(-1, 3, 4)
    prim = tris[:, 0, 3].copy().view(np.uint32)
    base = np.concatenate([[0], np.cumsum(sizes)])
    assert len(tris) == base[-1]
    for k, p in enumerate(meshes):
        seg = tris[base[k]:base[k + 1]]
        order = prim[base[k]:base[k + 1]]
        assert np.array_equal(np.sort(order), np.arange(sizes[k]))
        if device_blas:
            assert np.array_equal(order, np.arange(sizes[k]))
        assert seg[:, :, :3].tobytes() == p[order].tobytes()
    if not device_blas:
        _check_bvh(hs, int(base[-1]))
