"""The drop-in plugins through C++: tests/cpp/plugin_driver.cpp is compiled with g++
against the library and its mirror of the reference's plugin headers, loads scene files
through the plugin factory (XML -> Scene::activate -> Integrator::preprocess ->
Scene::render -> Integrator::render), and compares the camera film with a direct
gnd_gpu_render of the same passes bit for bit (sum wL, sum w). Covered: the path and
volpath plugins under their own names and under the reference's names (`path`,
`volpath`, the unchanged scene files), the default Gaussian film filter, and a render
cancelled from the progress callback."""
import subprocess

import pytest

from gianduia_b200 import scenes
from plugindriver import build_driver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    return build_driver(str(tmp_path_factory.mktemp("drv") / "plugin_driver"))


def _run(driver, xml, *extra):
    r = subprocess.run([driver, xml, *map(str, extra)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout
    return r.stdout


@pytest.mark.parametrize("integ", ["path_gpu", "path"])
def test_path_plugin(driver, tmp_path, integ):
    xml = scenes.cornell(str(tmp_path), width=48, height=40, spp=3, max_depth=6, integrator=integ)
    out = _run(driver, xml)
    assert "passes=3" in out


@pytest.mark.parametrize("integ", ["volpath_gpu", "volpath"])
def test_volpath_plugin(driver, tmp_path, integ):
    xml = scenes.volumetric(str(tmp_path), width=40, height=32, spp=2, max_depth=12, integrator=integ)
    _run(driver, xml)


def test_plugin_default_gaussian_filter(driver, tmp_path):
    """No <filter> in the scene file: the film takes the reference's default Gaussian."""
    xml = scenes.cornell(str(tmp_path), width=32, height=32, spp=2, filter="default")
    _run(driver, xml)


def test_plugin_cancel_from_callback(driver, tmp_path):
    """Integrator::cancel from the progress callback after pass 1 of 5: the film holds
    passes 0 and 1 and equals a direct render of those two."""
    xml = scenes.cornell(str(tmp_path), width=32, height=24, spp=5)
    out = _run(driver, xml, 1)
    assert "passes=2" in out
