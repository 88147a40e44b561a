"""High-spp CPU reference images for the relMSE gates of the image tests.

Each reference is the oracle (the CPU restatement of the reference render loop) at 4096
spp over a stated pixel window of one benchmark configuration:

  cornell     Cornell box, path, 256 x 256 (the whole image), depth 8, box filter
  volumetric  volumetric Cornell box, volpath, 512 x 512 scene, window [272, 400) x
              [208, 336) (the glass sphere and the medium around it), depth 32
  microfacet  microfacet grid, path, 1024 x 1024 scene, two 64 x 64 windows (among
              the brightest of the image; most of this scene is dark), depth 16

Passes [REF_PASS0, REF_PASS0 + 4096) key the reference's samples, so no test render
(which uses passes below 1,000,000) shares a sample with it. The images are computed
once and cached under baseline/_ref/relmse/ (not part of the repository: regenerate with
`python tests/relmse_refs.py`), each with a JSON record of its wall time and threads.
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CACHE = os.path.join(ROOT, "baseline", "_ref", "relmse")
REF_SPP = 4096
REF_PASS0 = 1 << 24

CONFIGS = {
    "cornell": dict(scene="cornell", kw=dict(width=256, height=256, spp=16, max_depth=8), windows=[(0, 0, 256, 256)]),
    "volumetric": dict(scene="volumetric", kw=dict(width=512, height=512, spp=64, max_depth=32),
                       windows=[(272, 208, 400, 336)]),
    "microfacet": dict(scene="microfacet", kw=dict(width=1024, height=1024, spp=64, max_depth=16, grid=64, seed=2),
                       windows=[(512, 512, 576, 576), (768, 384, 832, 448)]),
}


def scene_xml(name, out_dir):
    """Writes the configuration's scene file under out_dir; returns its path."""
    from gianduia_b200 import scenes
    cfg = CONFIGS[name]
    return getattr(scenes, cfg["scene"])(os.path.join(out_dir, name), **cfg["kw"])


def _path(name, k):
    return os.path.join(CACHE, "%s_w%d.npy" % (name, k))


def compute(name, out_dir, nthreads=0):
    """Renders the references of `name` with the oracle and writes them to the cache."""
    sys.path.insert(0, ROOT)
    from oracle import pyoracle as O
    os.makedirs(CACHE, exist_ok=True)
    xml = scene_xml(name, out_dir)
    sc = O.Scene.load(xml)
    rec = {"name": name, "spp": REF_SPP, "first_pass": REF_PASS0, "threads": nthreads or os.cpu_count(),
           "windows": [], "scene": CONFIGS[name]}
    for k, win in enumerate(CONFIGS[name]["windows"]):
        t = time.time()
        film = None
        paths = 0
        for s0 in range(REF_PASS0, REF_PASS0 + REF_SPP, 256):   # in chunks (float sums stay accurate)
            f, p, _ = sc.render(s0, s0 + 256, window=win, nthreads=nthreads)
            film = f.astype(np.float64) if film is None else film + f
            paths += p
        x0, y0, x1, y1 = win
        sub = film[y0:y1, x0:x1]
        img = np.where(sub[..., 3:4] > 0, sub[..., :3] / np.maximum(sub[..., 3:4], 1e-30), 0.0).astype(np.float32)
        np.save(_path(name, k), img)
        rec["windows"].append({"window": list(win), "paths": paths, "wall_s": time.time() - t,
                               "mean": float(img.mean())})
    with open(os.path.join(CACHE, name + ".json"), "w") as f:
        json.dump(rec, f, indent=1)
    return rec


def load(name):
    """The cached reference images of `name` (one per window), or None when not cached."""
    out = []
    for k in range(len(CONFIGS[name]["windows"])):
        p = _path(name, k)
        if not os.path.exists(p):
            return None
        out.append(np.load(p))
    return out


if __name__ == "__main__":
    import tempfile
    names = sys.argv[1:] or list(CONFIGS)
    d = tempfile.mkdtemp(prefix="gnd_relmse_")
    for n in names:
        r = compute(n, d)
        print(json.dumps({"name": n, "windows": r["windows"]}), flush=True)
