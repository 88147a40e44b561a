"""The reference-side plugin source shown in INTEGRATION.md compiles as it stands: the
code block of its "Reference-side binding" section is written to a file and compiled
with g++ against the library's mirror of the reference's plugin headers (the reference's
header names mapped onto hscene.h by tests/cpp/refshim). No GPU needed."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _binding_source():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    sec = text[text.index("## Reference-side binding"):]
    m = re.search(r"```cpp\n(.*?)```", sec, flags=re.S)
    assert m, "no C++ block in the binding section"
    return m.group(1)


def test_binding_sample_compiles(tmp_path):
    src = _binding_source()
    assert 'GND_REGISTER_CLASS(PathGpuIntegrator, "path_gpu")' in src
    assert "sceneFile" in src and "FileResolver::getBasePath()" in src
    f = tmp_path / "pathGpu.cpp"
    f.write_text(src)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [cxx, "-std=c++20", "-fsyntax-only", "-Wall", "-Werror=return-type",
           "-I", os.path.join(ROOT, "tests", "cpp", "refshim"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "gianduia_b200", "csrc", "include"),
           "-I", os.path.join(ROOT, "gianduia_b200", "csrc", "host"), str(f)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
