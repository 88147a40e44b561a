"""Builds tests/cpp/plugin_driver.cpp with g++ against the library (shared by the CPU and
GPU plugin tests)."""
import os
import subprocess

import gianduia_b200 as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_driver(out):
    lib = G._build.build()
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [cxx, "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "gianduia_b200", "csrc", "include"),
           "-I", os.path.join(ROOT, "gianduia_b200", "csrc", "host"),
           os.path.join(ROOT, "tests", "cpp", "plugin_driver.cpp"), lib,
           "-Wl,-rpath," + os.path.dirname(lib), "-pthread", "-o", out]
    subprocess.run(cmd, check=True)
    return out
