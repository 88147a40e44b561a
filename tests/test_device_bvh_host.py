"""Host side of the device-built mesh trees (GND_HOST_DEVICE_BLAS), no GPU: the scene
description keeps only the top-level tree, triangles in original order with the
identity original -> leaf map, mesh records that tile the triangles, and unset instance
roots for the upload to fill."""
import numpy as np

import gianduia_b200 as G
from gianduia_b200 import scenes

K_EMPTY = 0xFFFFFFFF


def test_triangle_soup_desc():
    tri = scenes.random_triangles(3000, seed=2)
    host = G.HostScene.from_triangles(tri)
    dev = G.HostScene.from_triangles(tri, device_blas=True)
    assert host.desc.blas_on_device == 0 and dev.desc.blas_on_device == 1
    # one instance: the top-level tree is one node; the host build adds the mesh tree
    assert dev.desc.num_nodes == 1 and host.desc.num_nodes > 100
    t = dev.tris()
    assert np.array_equal(t[:, 3].view(np.uint32), np.arange(3000, dtype=np.uint32))
    assert np.array_equal(t[:, [0, 1, 2, 4, 5, 6, 8, 9, 10]].reshape(-1, 3, 3), tri.reshape(-1, 3, 3))
    assert dev.inst_trav()[0, 13].view(np.uint32) == K_EMPTY
    # the host-built description is unchanged by the option's existence
    assert sorted(host.tris()[:, 3].view(np.uint32)) == list(range(3000))


def test_scene_file_desc(tmp_path):
    xml = scenes.cornell(str(tmp_path), width=16, height=16, spp=1)
    host = G.HostScene.load_xml(xml)
    dev = G.HostScene.load_xml(xml, device_blas=True)
    assert dev.desc.blas_on_device == 1
    assert dev.desc.num_tris == host.desc.num_tris and dev.desc.num_meshes == host.desc.num_meshes
    assert dev.desc.num_nodes < host.desc.num_nodes
    # the top-level tree is the same
    tl = host.tlas_list()
    assert np.array_equal(dev.tlas_list(), tl)
    assert np.array_equal(dev.nodes()[: dev.desc.num_nodes]["lo_hi"], host.nodes()[: dev.desc.num_nodes]["lo_hi"])
    # mesh records tile the triangles in order, the map is the identity
    import ctypes
    mr = np.frombuffer(ctypes.string_at(dev.desc.meshes, 16 * dev.desc.num_meshes), np.uint32).reshape(-1, 4)
    assert mr[0, 2] == 0 and np.array_equal(mr[1:, 2], np.cumsum(mr[:-1, 1]))
    assert int(mr[:, 1].sum()) == dev.desc.num_tris
    o2l = np.ctypeslib.as_array((ctypes.c_uint32 * dev.desc.orig_to_leaf_len).from_address(dev.desc.orig_to_leaf))
    assert np.array_equal(o2l, np.arange(dev.desc.num_tris, dtype=np.uint32))
    # mesh instances wait for their root; analytic shapes have none
    it = dev.inst_trav()
    kind = it[:, 12].view(np.uint32)
    assert (it[kind == 0, 13].view(np.uint32) == K_EMPTY).all()
