"""The drop-in plugins' C++ side without a GPU: the driver that loads scene files through
the plugin factory compiles against the library's mirror of the reference's plugin
headers, and with no CUDA device the plugin's preprocess fails loudly (no CPU fallback)."""
import subprocess

import pytest

from gianduia_b200 import scenes
from plugindriver import build_driver


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_driver_builds(tmp_path):
    exe = build_driver(str(tmp_path / "plugin_driver"))
    assert subprocess.run([exe], capture_output=True, text=True).returncode == 1   # usage


@pytest.mark.skipif(_gpu_present(), reason="a CUDA device is present")
def test_plugin_fails_loudly_without_device(tmp_path):
    exe = build_driver(str(tmp_path / "plugin_driver"))
    xml = scenes.cornell(str(tmp_path / "c"), width=16, height=16, spp=1, integrator="path")
    r = subprocess.run([exe, xml], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "gnd_gpu_create" in r.stdout and "no CUDA device" in r.stdout
