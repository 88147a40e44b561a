"""Builds gianduia_b200/_lib/libgianduia_b200.so: CUDA kernels for sm_100a (nvcc) and the
host scene framework (g++), linked into one shared library with the C ABI of
include/gnd_gpu.h.

Every translation unit is compiled without floating-point contraction (nvcc -fmad=false,
g++ -ffp-contract=off) so that geometry matches the reference's separately rounded
arithmetic bit for bit.

Usage: python -m gianduia_b200.build [--force] [--verbose-ptxas]
"""
import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(OUT_DIR, "libgianduia_b200.so")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
STAMP = os.path.join(OUT_DIR, "source.sha256")

NVCC = os.environ.get("GND_NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
# The system compiler (an environment override may point at a different libstdc++).
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
INCLUDES = ["-I", os.path.join(ROOT, "include"), "-I", os.path.join(CSRC, "include"), "-I", os.path.join(CSRC, "cuda")]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
              "-Xcompiler", "-fPIC", "-ccbin", CXX, "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++20", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-pthread", "-Wall", "-Wno-unused-variable"]


def sources():
    cu, cpp, hdr = [], [], []
    for d, _, files in os.walk(CSRC):
        for f in sorted(files):
            p = os.path.join(d, f)
            if f.endswith(".cu"):
                cu.append(p)
            elif f.endswith(".cpp"):
                cpp.append(p)
            elif f.endswith((".h", ".cuh")):
                hdr.append(p)
    hdr.append(os.path.join(ROOT, "include", "gnd_gpu.h"))
    return sorted(cu), sorted(cpp), sorted(hdr)


def source_hash():
    cu, cpp, hdr = sources()
    h = hashlib.sha256()
    for p in cu + cpp + hdr + [os.path.abspath(__file__)]:
        h.update(os.path.relpath(p, ROOT).encode())
        with open(p, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def up_to_date():
    if not os.path.exists(LIB) or not os.path.exists(STAMP):
        return False
    with open(STAMP) as f:
        return f.read().strip() == source_hash()


def _compile(src, verbose_ptxas=False):
    obj = os.path.join(OBJ_DIR, os.path.relpath(src, CSRC).replace(os.sep, "_") + ".o")
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + INCLUDES + (["-Xptxas", "-v"] if verbose_ptxas else []) + ["-c", src, "-o", obj]
    else:
        cmd = [CXX] + CXX_FLAGS + INCLUDES + ["-I", os.path.join(CSRC, "host"), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return obj, r.stderr


def build(force=False, verbose_ptxas=False, quiet=True):
    """Compiles and links the library when any source changed; returns its path."""
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    cu, cpp, _ = sources()
    logs = []
    with cf.ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
        futs = [ex.submit(_compile, s, verbose_ptxas) for s in cu + cpp]
        objs = []
        for f in futs:
            o, log = f.result()
            objs.append(o)
            if log:
                logs.append(log)
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-shared", "-ccbin", CXX, "-Xcompiler", "-fPIC", "-o", tmp] + objs + ["-cudart", "static", "-lpthread", "-lz"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    os.replace(tmp, LIB)
    with open(STAMP, "w") as f:
        f.write(source_hash())
    if not quiet or verbose_ptxas:
        sys.stderr.write("".join(logs))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force or a.verbose_ptxas, verbose_ptxas=a.verbose_ptxas, quiet=False))
