"""Thin-lens camera (thinLens.cpp:13-99) on the CPU: the oracle's polygon aperture warp
(warp.cpp:86-113), properties of its camera rays, and the host framework's camera record
for a `thinlens` scene. The images themselves are compared on the GPU
(test_gpu_camera.py)."""
import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes
from oracle import pyoracle as O

LENS_DOF = {"lens_radius": 0.12, "focal_distance": 3.0}


def polygon(u0, u1, blades):
    return O.warp(5, (u0, u1, float(blades)))[:2]


@pytest.mark.parametrize("blades", [3, 5, 6, 9])
def test_polygon_inside_and_uniform(blades):
    rng = np.random.default_rng(blades)
    u = rng.random((4000, 2)).astype(np.float32)
    p = np.array([polygon(a, b, blades) for a, b in u])
    # inside the regular polygon inscribed in the unit circle with a corner at the top:
    # the distance to the centre along each edge normal is at most cos(pi / blades)
    ang = np.pi / 2 + (np.arange(blades) + 0.5) * 2 * np.pi / blades
    normals = np.stack([np.cos(ang), np.sin(ang)], axis=1)
    assert (p @ normals.T).max() <= np.cos(np.pi / blades) + 1e-5
    # a corner at the top: (0, 1) is the far corner of the first blade (s.x just below
    # 1 / blades puts the point at radius ~1, s.y = 0 on that blade's first edge)
    assert np.allclose(polygon(0.999999 / blades, 0.0, blades), [0.0, 1.0], atol=1e-3)
    # uniform over the area: the mean is the centre, and each triangle gets 1/blades
    assert np.abs(p.mean(axis=0)).max() < 0.05
    sector = np.floor(((np.arctan2(p[:, 1], p[:, 0]) - np.pi / 2) % (2 * np.pi)) / (2 * np.pi / blades)).astype(int)
    counts = np.bincount(sector, minlength=blades)
    assert np.abs(counts / len(p) - 1 / blades).max() < 5 * np.sqrt((1 / blades) / len(p))


def test_polygon_below_three_blades_is_the_disk():
    for u in [(0.1, 0.2), (0.7, 0.9), (0.5, 0.5)]:
        assert np.array_equal(polygon(u[0], u[1], 2), O.warp(0, u)[:2])


def test_thin_lens_without_lens_equals_perspective(tmp_path):
    """lens_radius 0, k1 0 and no aberration: the thin-lens equations reduce to the
    perspective camera's operation for operation, so the rays are bit-identical."""
    a = O.Scene.load(scenes.cornell(str(tmp_path / "a"), width=24, height=16, spp=1))
    b = O.Scene.load(scenes.cornell(str(tmp_path / "b"), width=24, height=16, spp=1, lens={"vignetting": False}))
    py, px = np.mgrid[0:16, 0:24].astype(np.int32)
    ra = a.camera_rays(3, px.ravel(), py.ravel())
    rb = b.camera_rays(3, px.ravel(), py.ravel())
    assert np.array_equal(ra, rb)


def test_depth_of_field_rays_meet_at_the_focal_plane(tmp_path):
    """Each thin-lens ray leaves the lens disk and passes through the point where the
    pinhole ray of the same film position crosses the focal plane."""
    f = LENS_DOF["focal_distance"]
    pin = O.Scene.load(scenes.cornell(str(tmp_path / "a"), width=32, height=32, spp=1))
    lens = O.Scene.load(scenes.cornell(str(tmp_path / "b"), width=32, height=32, spp=1, lens=LENS_DOF))
    py, px = np.mgrid[0:32, 0:32].astype(np.int32)
    rp = pin.camera_rays(0, px.ravel(), py.ravel())
    rl = lens.camera_rays(0, px.ravel(), py.ravel())
    eye = np.array([0.0, 0.0, 3.5])
    view = np.array([0.0, 0.0, -1.0])          # the Cornell camera looks down -z
    dp = rp[:, 4:7].astype(np.float64)
    focus = eye + dp * (f / (dp @ view))[:, None]
    o, d = rl[:, 0:3].astype(np.float64), rl[:, 4:7].astype(np.float64)
    assert np.abs(o[:, 2] - 3.5).max() < 1e-6
    assert np.linalg.norm(o[:, :2], axis=1).max() <= LENS_DOF["lens_radius"] * (1 + 1e-5)
    assert np.linalg.norm(o - eye, axis=1).mean() > 0.3 * LENS_DOF["lens_radius"]
    to_focus = focus - o
    cross = np.linalg.norm(np.cross(to_focus / np.linalg.norm(to_focus, axis=1)[:, None], d), axis=1)
    assert cross.max() < 1e-5
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)


def test_host_camera_record(tmp_path):
    lens = {"lens_radius": 0.05, "focal_distance": 2.5, "k1": 0.1, "ca_axial": 0.02, "ca_lateral": 0.01,
            "vignetting": True, "blades": 6}
    cam = G.HostScene.load_xml(scenes.cornell(str(tmp_path / "a"), width=40, height=20, spp=1, lens=lens)).camera()
    assert cam["kind"] == 1 and cam["blades"] == 6 and cam["vignetting"] == 1
    for k in ("lens_radius", "focal_distance", "k1", "ca_axial", "ca_lateral"):
        assert cam[k] == np.float32(lens[k]), k
    assert cam["width"] == 40 and cam["height"] == 20 and cam["aspect"] == np.float32(2.0)
    assert np.allclose(cam["origin"], [0.0, 0.0, 3.5])
    pin = G.HostScene.load_xml(scenes.cornell(str(tmp_path / "b"), width=40, height=20, spp=1)).camera()
    assert pin["kind"] == 0 and pin["lens_radius"] == 0.0
    # the pinhole part of the record is the same for both camera types
    assert np.array_equal(pin["to_world"], cam["to_world"]) and pin["scale"] == cam["scale"]
    # a malformed integer reads as 0, as the reference parser's as_int does
    # (parser.cpp:62-64): six "blades" become none, the disk aperture
    bad = scenes.cornell(str(tmp_path / "c"), width=8, height=8, spp=1, lens={"blades": 6})
    with open(bad) as fh:
        text = fh.read().replace('<integer name="blades" value="6"/>', '<integer name="blades" value="six"/>')
    with open(bad, "w") as fh:
        fh.write(text)
    cam = G.HostScene.load_xml(bad).camera()
    assert cam["kind"] == 1 and cam["blades"] == 0
