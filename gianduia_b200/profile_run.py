"""Small fixed workloads for profiler captures (ncu), sized to end in seconds:

  python -m gianduia_b200.profile_run trace     closest-hit batch of the traversal
                                                micro-benchmark: 2^20 triangles, 2^22 rays
  python -m gianduia_b200.profile_run render    one 1-spp pass of the 1024x1024
                                                microfacet render (path_gpu, depth 16)
  python -m gianduia_b200.profile_run batched [spp]
                                                the microfacet render in batched mode,
                                                `spp` passes (default 1) sharing the pool
  python -m gianduia_b200.profile_run volpath [spp] [batched]
                                                the 512x512 volumetric Cornell box
                                                (volpath_gpu, depth 32), `spp` passes
                                                (default 1), plain unless `batched`
  python -m gianduia_b200.profile_run all       trace, then render

Arguments of the form name=value (gnd_tune fields, e.g. ray_sort=3) set the rendered
scene's engine settings; `gaussian` renders the microfacet scene with the reference's
default Gaussian film filter (radius 2, alpha 2) instead of its box filter.
"""
import os
import sys
import tempfile

import gianduia_b200 as G
from gianduia_b200 import scenes


def run_trace(ctx, tune=None):
    tri = scenes.random_triangles(1 << 20, seed=1)
    rays = scenes.random_rays(1 << 22, seed=1)
    sid = ctx.upload(G.HostScene.from_triangles(tri))
    if tune:
        ctx.set_tune(sid, **tune)
    h = ctx.trace_closest(sid, rays)
    print("trace: %d of %d rays hit" % (int((h["inst"] >= 0).sum()), rays.shape[0]))
    ctx.free_scene(sid)


def run_render(ctx, batched=False, spp=1, tune=None, gaussian=False):
    xml = scenes.microfacet(os.path.join(tempfile.gettempdir(), "gnd_bench_microfacet_r0"), width=1024, height=1024,
                            spp=64, max_depth=16, grid=64, seed=2)
    hs = G.HostScene.load_xml(xml)
    if gaussian:
        d = hs.desc
        d.filter, d.filter_radius[0], d.filter_radius[1], d.filter_alpha = 1, 2.0, 2.0, 2.0
    sid = ctx.upload(hs)
    if tune:
        ctx.set_tune(sid, **tune)
    _, st = ctx.render(sid, spp=spp, batched=batched)
    print("render:", st)
    ctx.free_scene(sid)


def run_volpath(ctx, spp=1, batched=False, tune=None):
    xml = scenes.volumetric(os.path.join(tempfile.gettempdir(), "gnd_prof_volumetric"), width=512, height=512, spp=64,
                            max_depth=32)
    sid = ctx.upload(G.HostScene.load_xml(xml))
    if tune:
        ctx.set_tune(sid, **tune)
    _, st = ctx.render(sid, spp=spp, batched=batched)
    print("volpath:", st)
    ctx.free_scene(sid)


def main(argv):
    tune = {k: int(v) for k, v in (a.split("=", 1) for a in argv[1:] if "=" in a)}
    gaussian = "gaussian" in argv
    argv = [a for a in argv if "=" not in a and a != "gaussian"]
    what = argv[1] if len(argv) > 1 else "all"
    ctx = G.GpuContext(0)
    if what in ("trace", "all"):
        run_trace(ctx, tune=tune)
    if what in ("render", "all"):
        run_render(ctx, tune=tune)
    if what == "batched":
        run_render(ctx, batched=True, spp=int(argv[2]) if len(argv) > 2 else 1, tune=tune, gaussian=gaussian)
    if what == "volpath":
        run_volpath(ctx, spp=int(argv[2]) if len(argv) > 2 else 1, batched=len(argv) > 3 and argv[3] == "batched",
                    tune=tune)
    ctx.close()


if __name__ == "__main__":
    main(sys.argv)
