"""Benchmark of the B200 radiance path (path_gpu wavefront integrator).

Workload (one step = one full render): the microfacet scene -- 1024x1024, 64 spp,
path max depth 16, ground quad plus a 64x64 grid of displaced icospheres
(5,242,880 + 2 triangles, 4105 instances) with plastic / rough conductor / rough glass
and 8 spherical emitters; synthetic, seeded (gianduia_b200/scenes.py).

Metric: Mpaths/s (camera samples per second, whole job). N GPUs: weak scaling over the
sample passes -- rank r renders passes [r*64, (r+1)*64) of the same image and the exact
films (fixed-point sums of wL and w, plus sum wL^2) are reduced to rank 0 (the sharded
render's only exchange), where they equal one render of all N*64 passes bit for bit.
The timed steps run the production path (per-bounce loop replayed as CUDA graphs); the
roofline's extend-kernel time comes from a separate instrumented render.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the CPU restatement of the reference's render loop (the
reference itself cannot be built here) on this host's cores, one pass of the same
image per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpaths/s at matched relMSE; serve p50/p99 time-to-image vs plain GPU"
# how the CPU restatement of the reference (the oracle, also the timed CPU baseline) is built
CPU_BUILD = ("g++ -O3 -march=x86-64-v3 -ffp-contract=off; 4-lane slab and Moller-Trumbore loops vectorised "
             "(the reference's Highway lanes); one std::thread per host core over image rows")
CPU_NOTE = ("a C++ port of the reference's render loop, not the reference binary (its glm / Highway / TBB / "
            "vcpkg build cannot be compiled here): GPU/CPU ratios are against this port")
WORKLOAD = dict(width=1024, height=1024, spp=64, max_depth=16, grid=64, seed=2)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def scene_dir(rank):
    d = os.environ.get("GND_SCENE_DIR") or os.path.join(tempfile.gettempdir(), "gnd_bench_microfacet_r%d" % rank)
    return d


def make_scene(rank):
    from gianduia_b200 import scenes
    t = time.time()
    p = scenes.microfacet(scene_dir(rank), **WORKLOAD)
    log("scene ready in %.1fs: %s" % (time.time() - t, p))
    return p


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception as e:
            log("clock sampling unavailable:", e)
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(xml, seconds=12.0):
    """The oracle (CPU restatement of the reference render loop) on this host's cores:
    full-image passes of the same scene until `seconds` of render time have elapsed."""
    from oracle import pyoracle as O
    t = time.time()
    sc = O.Scene.load(xml)
    log("oracle scene load %.1fs" % (time.time() - t))
    paths = 0
    el = 0.0
    s = 0
    while el < seconds and s < WORKLOAD["spp"]:
        t = time.perf_counter()
        _, p, _ = sc.render(s, s + 1)
        el += time.perf_counter() - t
        paths += p
        s += 1
    cores = os.cpu_count() or 1
    return {"value": paths / el / 1e6, "unit": "Mpaths/s", "cores": cores, "kind": "port",
            "build": CPU_BUILD, "note": CPU_NOTE,
            "sample": "%d full-image passes (%d paths) of the 1024x1024 microfacet scene" % (s, paths)}


def run_reference(args, rank, world):
    if rank != 0:
        return
    xml = make_scene(0)
    from oracle import pyoracle as O
    sc = O.Scene.load(xml)
    cores = os.cpu_count() or 1
    for w in range(args.warmup):
        sc.render(10000 + w, 10001 + w)
    times, paths = [], 0
    for k in range(args.steps):
        t = time.perf_counter()
        _, p, _ = sc.render(k, k + 1)
        times.append(time.perf_counter() - t)
        paths += p
    total = sum(times)
    v = paths / total / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, gianduia_b200/scenes.py)",
            "config": {"workload": "microfacet 1024x1024 path depth 16, one full-image pass (1,048,576 paths) per step",
                       "l2": "scene (0.7 GB) larger than L2"},
            "cpu_baseline": {"value": v, "unit": "Mpaths/s", "cores": cores, "kind": "port", "build": CPU_BUILD,
                             "note": CPU_NOTE, "sample": "one 1024x1024 pass per step, %d steps" % args.steps},
            "e2e": {"value": v, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def traversal_leg(ctx):
    """The traversal micro-benchmark: 2^20 random triangles (one mesh, the host SAH BVH4),
    2^24 random rays with tmax = inf, closest hit and any hit on device buffers, timed with
    CUDA events on the launching stream (median of 5 after 2 warm-ups). Also measures the
    read bandwidth of L2 (32 MiB buffer) and HBM (4 GiB buffer) for the roofline."""
    import torch
    import gianduia_b200 as G
    from gianduia_b200 import scenes
    n = 1 << 24
    tri = scenes.random_triangles(1 << 20, seed=1)
    rays = scenes.random_rays(n, seed=1)
    hs = G.HostScene.from_triangles(tri)
    sid = ctx.upload(hs)
    dr = torch.from_numpy(rays).cuda()
    dh = torch.empty((n, 5), dtype=torch.int32, device="cuda")
    docc = torch.empty(n, dtype=torch.uint8, device="cuda")
    strm = torch.cuda.Stream()
    st = strm.cuda_stream
    out = {"workload": "2^20 random triangles (centroids U[0,1]^3, vertex offsets N(0, 0.01^2)), 2^24 rays "
                       "(origins U[-0.5,1.5]^3, uniform directions, tmax inf)"}
    closest = lambda: ctx.trace_closest_dev(sid, dr.data_ptr(), n, dh.data_ptr(), st)
    anyhit = lambda: ctx.trace_any_dev(sid, dr.data_ptr(), n, docc.data_ptr(), st)
    # default settings (trace_leaf_batch 12); the full node phase of every warp
    # (trace_leaf_batch 32, the earlier default); the batch traversed in ray-key order
    # (ray_sort bit 2, the reordering inside the timed region)
    runs = [("closest", closest, {}), ("any", anyhit, {}),
            ("closest_full_node_phase", closest, {"trace_leaf_batch": 32}),
            ("any_full_node_phase", anyhit, {"trace_leaf_batch": 32}),
            ("closest_key_order", closest, {"ray_sort": 4}), ("any_key_order", anyhit, {"ray_sort": 4})]
    for name, fn, tune_fields in runs:
        ctx.set_tune(sid, **dict({"ray_sort": 0, "trace_leaf_batch": 12}, **tune_fields))
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(strm)
            fn()
            e1.record(strm)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = float(statistics.median(ts))
        out[name + "_ms"] = ms
        out[name + "_mrays_s"] = n / ms / 1e3
    ctx.set_tune(sid, ray_sort=0, trace_leaf_batch=12)
    nodes = torch.zeros(n, dtype=torch.int32, device="cuda")
    tris = torch.zeros(n, dtype=torch.int32, device="cuda")
    ctx.trace_count_dev(sid, dr.data_ptr(), n, nodes.data_ptr(), tris.data_ptr(), st)
    torch.cuda.synchronize()
    npr, tpr = float(nodes.double().sum()) / n, float(tris.double().sum()) / n
    bytes_per_ray = npr * 128 + tpr * 48 + 32 + 20
    achieved = bytes_per_ray * n / (out["closest_ms"] * 1e-3) / 1e9
    l2 = max(ctx.read_bandwidth(32 << 20, 200), ctx.read_bandwidth(64 << 20, 100))
    hbm = ctx.read_bandwidth(4 << 30, 3)
    scene_bytes = ctx.scene_bytes(sid)
    out.update({"nodes_per_ray": npr, "tris_per_ray": tpr, "bytes_per_ray": bytes_per_ray,
                "closest_achieved_gbs": achieved, "l2_read_gbs": l2, "hbm_read_gbs": hbm,
                "scene_bytes": scene_bytes, "frac_of_l2": achieved / l2, "frac_of_hbm": achieved / hbm,
                "bound": "l2" if scene_bytes < 100e6 else "hbm",
                "hit_frac": float((dh[:, 3] >= 0).float().mean().item())})
    ctx.free_scene(sid)
    del dr, dh, docc, nodes, tris
    torch.cuda.empty_cache()
    out["key_order_closest_achieved_gbs"] = bytes_per_ray * n / (out["closest_key_order_ms"] * 1e-3) / 1e9
    out["key_order_frac_of_l2"] = out["key_order_closest_achieved_gbs"] / l2
    log("traversal: closest %.0f Mrays/s (full node phases %.0f, key order %.0f), any %.0f Mrays/s (%.0f, %.0f); "
        "%.1f nodes %.1f tris per ray; %.0f GB/s = %.2f of L2 %.0f GB/s" % (
            out["closest_mrays_s"], out["closest_full_node_phase_mrays_s"], out["closest_key_order_mrays_s"],
            out["any_mrays_s"], out["any_full_node_phase_mrays_s"], out["any_key_order_mrays_s"],
            npr, tpr, achieved, achieved / l2, l2))
    return out


def device_bvh_leg(ctx, xml, host_sid, host_load_s, tune):
    """Mesh trees built on the GPU at upload against the host SAH build, on the bench
    scene (4105 meshes, 5.2M triangles) and on the traversal workload (one mesh of 2^20
    triangles): host load time without the mesh builds, upload wall time and the device
    build time (CUDA events), and the traversal / render speed through each tree."""
    import torch
    import gianduia_b200 as G
    from gianduia_b200 import scenes
    out = {}
    t = time.perf_counter()
    hd = G.HostScene.load_xml(xml, device_blas=True)
    out["host_load_s"] = time.perf_counter() - t
    out["host_load_sah_s"] = host_load_s
    hd.pin(True)
    ups, builds = [], []
    for k in range(4):
        t = time.perf_counter()
        sid = ctx.upload(hd)
        up = time.perf_counter() - t
        info = ctx.scene_info(sid)
        if k:
            ups.append(up)
            builds.append(info["build_ms"])
        if k < 3:
            ctx.free_scene(sid)
    hd.pin(False)
    out["upload_ms"] = 1e3 * statistics.median(ups)
    out["build_ms"] = statistics.median(builds)
    out["nodes"] = info["num_nodes"]
    ctx.set_tune(sid, **tune)
    film = np.zeros((hd.height, hd.width, 7), np.float32)
    for name, s in (("device_tree", sid), ("host_tree", host_sid)):
        ctx.render(s, spp=8, batched=True, film=film)
        ts = []
        for _ in range(3):
            _, st = ctx.render(s, spp=16, batched=True, film=film)
            ts.append(st["ms"])
        out[name + "_mpaths_s"] = st["paths"] / (statistics.median(ts) / 1e3) / 1e6
        _, cst = ctx.render(s, spp=2, profile=2)
        out[name + "_nodes_per_ray"] = cst["extend_nodes"] / max(1, cst["extend_rays"])
        out[name + "_tris_per_ray"] = cst["extend_tris"] / max(1, cst["extend_rays"])
    ctx.free_scene(sid)
    # one large mesh: the traversal workload
    n = 1 << 22
    tri = scenes.random_triangles(1 << 20, seed=1)
    rays = scenes.random_rays(n, seed=1)
    dr = torch.from_numpy(rays).cuda()
    dh = torch.empty((n, 5), dtype=torch.int32, device="cuda")
    strm = torch.cuda.Stream()
    for name, dev in (("soup_device_tree", True), ("soup_host_tree", False)):
        t = time.perf_counter()
        hs = G.HostScene.from_triangles(tri, device_blas=dev)
        host_s = time.perf_counter() - t
        t = time.perf_counter()
        s = ctx.upload(hs)
        up = time.perf_counter() - t
        ctx.trace_closest_dev(s, dr.data_ptr(), n, dh.data_ptr(), strm.cuda_stream)
        torch.cuda.synchronize()
        ts = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(strm)
            ctx.trace_closest_dev(s, dr.data_ptr(), n, dh.data_ptr(), strm.cuda_stream)
            e1.record(strm)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        out[name] = {"host_s": host_s, "upload_ms": up * 1e3, "build_ms": ctx.scene_info(s)["build_ms"],
                     "closest_mrays_s": n / statistics.median(ts) / 1e3}
        if dev:
            # refit of the same mesh to moved positions (device time of the refit kernels;
            # the first refit also walks the tree once)
            moved = tri.reshape(-1, 9) * np.float32(1.01) + np.float32(0.001)
            first = ctx.refit_mesh(s, 0, moved)
            out[name]["refit_ms"] = statistics.median([ctx.refit_mesh(s, 0, moved if k % 2 else tri) for k in range(4)])
            out[name]["first_refit_ms"] = first
        ctx.free_scene(s)
        hs.close()
    del dr, dh
    torch.cuda.empty_cache()
    log("device trees: host load %.2fs (SAH %.2fs), upload %.1f ms with a %.1f ms build; render %.0f vs %.0f Mpaths/s "
        "(%.1f vs %.1f nodes/ray); 2^20-triangle mesh built in %.1f ms (refit %.2f ms), %.0f vs %.0f Mrays/s" % (
            out["host_load_s"], host_load_s, out["upload_ms"], out["build_ms"], out["device_tree_mpaths_s"],
            out["host_tree_mpaths_s"], out["device_tree_nodes_per_ray"], out["host_tree_nodes_per_ray"],
            out["soup_device_tree"]["build_ms"], out["soup_device_tree"]["refit_ms"], out["soup_device_tree"]["closest_mrays_s"],
            out["soup_host_tree"]["closest_mrays_s"]))
    return out


def scenes_leg(ctx):
    """The two other render configurations at their full sizes: Cornell box (path, 256^2,
    16 spp, depth 8) and volumetric Cornell box (volpath, 512^2, 64 spp, depth 32), batched
    and plain, each the median of 3 renders after 1 warm-up (host wall time of the call);
    and the Cornell box with no <filter>, i.e. the reference's default Gaussian film
    filter (radius 2: every sample reaches up to 16 pixels)."""
    import gianduia_b200 as G
    from gianduia_b200 import scenes
    base = os.path.join(tempfile.gettempdir(), "gnd_bench_scenes")
    out = {}
    for name, xml in (("cornell", scenes.cornell(os.path.join(base, "cornell"))),
                      ("cornell_gaussian", scenes.cornell(os.path.join(base, "cornell_g"), filter="default")),
                      ("volumetric", scenes.volumetric(os.path.join(base, "volumetric")))):
        hs = G.HostScene.load_xml(xml)
        sid = ctx.upload(hs)
        film = np.zeros((hs.height, hs.width, 7), np.float32)
        rec = {"width": hs.width, "height": hs.height, "spp": hs.spp, "max_depth": hs.desc.max_depth,
               "integrator": ["path_gpu", "volpath_gpu"][hs.desc.integrator],
               "filter": ["box", "gaussian"][hs.desc.filter]}
        for mode in ("batched", "plain"):
            ts = []
            for k in range(4):
                t = time.perf_counter()
                _, st = ctx.render(sid, batched=(mode == "batched"), film=film)
                if k:
                    ts.append(time.perf_counter() - t)
            rec[mode + "_mpaths_s"] = st["paths"] / statistics.median(ts) / 1e6
        ctx.free_scene(sid)
        out[name] = rec
        log("%s: batched %.1f Mpaths/s, plain %.1f Mpaths/s" % (name, rec["batched_mpaths_s"], rec["plain_mpaths_s"]))
    return out


def cold_request_leg(ctx, xml, spp):
    """Time-to-image of a cold request: from the scene file on disk to the film in host
    memory -- parse and load the 4,105 OBJ files, build (mesh trees on the GPU, or the
    host SAH build), upload, render all passes batched, read the film back -- host wall
    time, median of 3 (the files sit in the OS page cache, as for a server that keeps
    receiving the same scenes)."""
    import gianduia_b200 as G
    out = {}
    for name, dev in (("device_trees", True), ("host_trees", False)):
        parts = []
        for _ in range(3):
            t0 = time.perf_counter()
            hs = G.HostScene.load_xml(xml, device_blas=dev)
            t1 = time.perf_counter()
            sid = ctx.upload(hs)
            t2 = time.perf_counter()
            ctx.render(sid, spp=spp, batched=True)
            t3 = time.perf_counter()
            ctx.free_scene(sid)
            hs.close()
            parts.append((t3 - t0, t1 - t0, t2 - t1, t3 - t2))
        tot, load, up, ren = sorted(parts)[1]
        out[name] = {"total_s": tot, "host_load_s": load, "upload_s": up, "render_and_readback_s": ren}
    log("cold request (file -> film): %.2f s with device-built trees, %.2f s with the host build" % (
        out["device_trees"]["total_s"], out["host_trees"]["total_s"]))
    return out


def gaussian_leg(ctx, hs, tune, spp):
    """The headline render with the reference's default film filter instead of the box:
    the same microfacet scene description uploaded with a Gaussian filter (radius 2,
    alpha 2; film.cpp:29), batched, median of 3 renders (device time)."""
    d = hs.desc
    saved = (d.filter, d.filter_radius[0], d.filter_radius[1], d.filter_alpha)
    d.filter, d.filter_radius[0], d.filter_radius[1], d.filter_alpha = 1, 2.0, 2.0, 2.0
    try:
        sid = ctx.upload(hs)
    finally:
        d.filter, d.filter_radius[0], d.filter_radius[1], d.filter_alpha = saved
    ctx.set_tune(sid, **tune)
    film = np.zeros((hs.height, hs.width, 7), np.float32)
    ctx.render(sid, spp=spp, batched=True, film=film)
    ts = []
    for _ in range(3):
        _, st = ctx.render(sid, spp=spp, batched=True, film=film)
        ts.append(st["ms"])
    ctx.free_scene(sid)
    ms = statistics.median(ts)
    log("microfacet with the Gaussian film filter: %.1f ms, %.1f Mpaths/s" % (ms, st["paths"] / ms / 1e3))
    return {"filter": "gaussian radius 2 alpha 2 (the reference's default)", "ms": ms,
            "mpaths_s": st["paths"] / (ms / 1e3) / 1e6}


def serve_leg(ctx, microfacet_sid, n_requests, n_policy=300):
    """The serving stream: requests over {Cornell box, microfacet grid, volumetric Cornell
    box} with Poisson arrivals at 80% of the job server's capacity, served by the job
    server and, for comparison, one at a time by plain renders in arrival order.
    Capacity: 200 requests of the same distribution submitted at once (samples/s), so
    that the arrival rate offers 0.8 x capacity for the stream's own mean request size.
    The FIFO and SRPT hand-out policies are compared on the first `n_policy` requests."""
    import gianduia_b200 as G
    from gianduia_b200 import scenes, serving
    base = os.path.join(tempfile.gettempdir(), "gnd_bench_serve")
    sids = {"microfacet": microfacet_sid,
            "cornell": ctx.upload(G.HostScene.load_xml(scenes.cornell(os.path.join(base, "cornell")))),
            "volumetric": ctx.upload(G.HostScene.load_xml(scenes.volumetric(os.path.join(base, "volumetric"))))}
    integ = {"microfacet": 0, "cornell": 0, "volumetric": 1}
    ctx.set_hbm_budget(150 * 10**9)   # the stream's HBM admission budget
    ctx.serve_policy("deadline")
    t = time.perf_counter()
    cap_rps, cap_sps = serving.calibrate_capacity(ctx, sids, integ, n=200)
    log("serve: capacity %.1f Mpaths/s (%.2f req/s) from 200 requests at once, %.1fs" % (
        cap_sps / 1e6, cap_rps, time.perf_counter() - t))
    reqs = serving.make_requests(n_requests, seed=4)
    total = sum(serving.samples(r) for r in reqs)
    rate = 0.8 * cap_sps / (total / n_requests)   # offered load 0.8 for this stream's mean request
    arrivals = serving.poisson_arrivals(n_requests, rate, seed=4)
    t = time.perf_counter()
    lat, makespan = serving.run_served(ctx, sids, integ, reqs, arrivals)
    log("serve: %d requests served in %.1fs" % (n_requests, time.perf_counter() - t))
    other = {}
    npol = min(n_policy, n_requests)
    for pol in ("fifo", "srpt", "deadline"):
        ctx.serve_policy(pol)
        other[pol] = serving.latency_stats(serving.run_served(ctx, sids, integ, reqs[:npol], arrivals[:npol])[0])
    ctx.serve_policy("deadline")
    t = time.perf_counter()
    service, model = serving.plain_service_model(ctx, sids, integ, reqs)
    log("serve: plain render-time model over %d (scene, resolution, depth) keys in %.1fs, largest error %s" % (
        model["keys"], time.perf_counter() - t, model["max_rel_err"]))
    plain_lat = serving.fifo_finish(arrivals, service) - arrivals
    s, p = serving.latency_stats(lat), serving.latency_stats(plain_lat)
    for k in ("cornell", "volumetric"):
        ctx.free_scene(sids[k])
    log("serve: %d requests at %.2f req/s; p50 %.3f s p99 %.3f s (plain one at a time: p50 %.3f s p99 %.3f s)" % (
        n_requests, rate, s["p50"], s["p99"], p["p50"], p["p99"]))
    plain_sps = total / float(service.sum())
    return {"requests": n_requests, "arrivals": "poisson, seed 4",
            "policy": "deadline (submission + 4x estimated render time, earliest first)",
            "rate_rps": rate, "capacity_rps": cap_rps, "capacity_mpaths_s": cap_sps / 1e6,
            "capacity_from": "200 requests of the stream's distribution submitted at once",
            "offered_load": rate * (total / n_requests) / cap_sps,
            "p50_s": s["p50"], "p99_s": s["p99"], "mean_s": s["mean"], "max_s": s["max"],
            "plain_p50_s": p["p50"], "plain_p99_s": p["p99"], "plain_mean_s": p["mean"],
            "p50_speedup": p["p50"] / s["p50"], "p99_speedup": p["p99"] / s["p99"],
            "served_mpaths_s": total / makespan / 1e6, "makespan_s": makespan,
            "plain_mpaths_s": plain_sps / 1e6, "capacity_vs_plain": cap_sps / plain_sps,
            "policies_first_requests": npol,
            "fifo_p50_s": other["fifo"]["p50"], "fifo_p99_s": other["fifo"]["p99"],
            "srpt_p50_s": other["srpt"]["p50"], "srpt_p99_s": other["srpt"]["p99"],
            "deadline_p50_s": other["deadline"]["p50"], "deadline_p99_s": other["deadline"]["p99"],
            "plain_model": model,
            "note": "plain time-to-image: the FIFO recurrence over plain render times, each the fixed + spp x "
                    "per-pass time measured for its (scene, resolution, depth) (plain renders run their passes "
                    "one after another); served_mpaths_s at 80% offered load is bounded by the arrivals"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--plain", action="store_true", help="one pass in flight (no refill) for the timed steps")
    ap.add_argument("--no-traversal", action="store_true", help="skip the traversal micro-benchmark")
    ap.add_argument("--no-autotune", action="store_true", help="render with the default engine settings")
    ap.add_argument("--no-scenes", action="store_true", help="skip the Cornell / volumetric renders")
    ap.add_argument("--no-device-bvh", action="store_true", help="skip the device tree build measurements")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="requests in the serving stream (2000: the full stream); 0 skips it")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import gianduia_b200 as G
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)

    xml = make_scene(rank)
    t = time.time()
    hs = G.HostScene.load_xml(xml)
    host_load_s = time.time() - t
    log("host load + BVH build %.1fs (%d tris, %d nodes, %d instances)" % (
        host_load_s, hs.desc.num_tris, hs.desc.num_nodes, hs.desc.num_instances))
    ctx = G.GpuContext(local)
    sid = ctx.upload(hs)
    scene_bytes = ctx.scene_bytes(sid)
    from gianduia_b200.sharding import as_int64, as_uint64, pass_range, reduce_fixed_film
    spp = WORKLOAD["spp"]
    first, _ = pass_range(rank, world, spp)
    npix = WORKLOAD["width"] * WORKLOAD["height"]

    # traversal work of the extend kernel (instrumented run on the same paths)
    _, cst = ctx.render(sid, spp=8, first_pass=first, profile=2)
    nodes_per_ray = cst["extend_nodes"] / max(1, cst["extend_rays"])
    tris_per_ray = cst["extend_tris"] / max(1, cst["extend_rays"])
    log("extend work: %.2f nodes, %.2f triangles per ray" % (nodes_per_ray, tris_per_ray))

    batched = not args.plain
    tune = ctx.get_tune(sid)
    if not args.no_autotune:
        t = time.time()
        tune, tune_mp = ctx.autotune(sid, spp=32, budget_ms=16000)
        log("autotune %.1fs: %s (%.0f Mpaths/s at 32 spp)" % (time.time() - t, tune, tune_mp))
    # one host film buffer for every render of the run (each render adds its sums into it)
    film = np.zeros((WORKLOAD["height"], WORKLOAD["width"], 7), np.float32)
    for w in range(args.warmup):
        ctx.render(sid, spp=spp, first_pass=first, batched=batched, film=film)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    reduced = []

    def step(profile=0):
        """One full render of this rank's passes; with N > 1 the exact films (fixed-point
        sums) are reduced to rank 0, which keeps the result."""
        if not dist:
            return ctx.render(sid, spp=spp, first_pass=first, profile=profile, batched=batched, film=film)[1]
        fsum, fsq, st = ctx.render_fixed(sid, spp=spp, first_pass=first, profile=profile, batched=batched)
        ts, tq = torch.from_numpy(as_int64(fsum)).cuda(), torch.from_numpy(fsq).cuda()
        reduce_fixed_film(ts, tq, dist)
        if rank == 0:
            reduced[:] = [ts, tq]
        return st

    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    t0 = time.perf_counter()
    stats = []
    for k in range(args.steps):
        # the production path: CUDA-graph bounce loop, no per-launch instrumentation
        stats.append(step())
    barrier()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    dev_ms = sum(s["ms"] for s in stats)
    elapsed = max(wall, dev_ms / 1000.0)
    if dist:
        tt = torch.tensor([elapsed], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        elapsed = float(tt.item())
    paths_total = sum(s["paths"] for s in stats) * world
    value = paths_total / elapsed / 1e6
    rays = sum(s["rays"] for s in stats)
    # the roofline's extend time: a separate instrumented render of the same passes, each
    # extend launch bracketed by CUDA events on the engine's stream (graphs off in it)
    inst = ctx.render(sid, spp=spp, first_pass=first, profile=1, batched=batched,
                      film=np.zeros_like(film))[1]
    ext_rays, ext_ms, iters = inst["extend_rays"], inst["extend_ms"], inst["iterations"]
    film_check = None
    if dist and rank == 0 and reduced:
        fs = as_uint64(reduced[0].cpu().numpy())
        img = fs[..., :3].astype(np.float64) / np.maximum(fs[..., 3:4].astype(np.float64), 1.0)
        film_check = {"passes": spp * world, "mean_radiance": float(img.mean()),
                      "sum_w": int(fs[..., 3].sum(dtype=np.uint64)) / 16777216.0}

    # e2e through the C ABI with host buffers: scene upload from pinned host memory +
    # render + film read-back to host memory: the resolved float film (sum wL rgb, sum w,
    # sum wL^2 rgb) per pixel, or with N > 1 the exact film (4 x uint64 + 3 x float)
    film_bytes = npix * 7 * 4 if not dist else npix * (4 * 8 + 3 * 4)

    def timed_upload(hscene):
        t = time.perf_counter()
        s = ctx.upload(hscene)
        return s, time.perf_counter() - t

    def e2e_run(hscene, label, overlap):
        """K steps, each uploading its own copy of the scene, rendering it, reading the film
        back and freeing the copy. With overlap, the upload of step k + 1 runs on a second
        host thread during step k's render (gnd_gpu_scene_upload copies on its own stream),
        as a renderer fed a stream of scenes would run; every upload is inside the timed
        region either way."""
        steps = 0 if args.no_e2e else max(1, args.steps)
        if not steps:
            return None
        hscene.pin(True)
        # untimed warm-up uploads of the freshly page-locked description (the renders are
        # warm from the device-timed steps)
        for _ in range(max(1, args.warmup)):
            s, _ = timed_upload(hscene)
            ctx.free_scene(s)
        pool = ThreadPoolExecutor(max_workers=1) if overlap else None
        barrier()
        t0 = time.perf_counter()
        nxt, up_s = timed_upload(hscene)
        for k in range(steps):
            sid2 = nxt
            ctx.set_tune(sid2, **tune)
            pending = pool.submit(timed_upload, hscene) if (pool and k + 1 < steps) else None
            t_r = time.perf_counter()
            if dist:
                fsum, fsq, st = ctx.render_fixed(sid2, spp=spp, first_pass=first, batched=batched)
                reduce_fixed_film(torch.from_numpy(as_int64(fsum)).cuda(), torch.from_numpy(fsq).cuda(), dist)
            else:
                _, st = ctx.render(sid2, spp=spp, first_pass=first, batched=batched, film=film)
            t_re = time.perf_counter()
            if pending is not None:
                nxt, up_next = pending.result()
            elif k + 1 < steps:
                nxt, up_next = timed_upload(hscene)
            t_w = time.perf_counter()
            ctx.free_scene(sid2)
            log("e2e step (%s): upload %.1f ms%s, render %.1f ms, wait %.1f ms, free %.1f ms" % (
                label, up_s * 1e3, " (during the previous render)" if overlap and k else "", (t_re - t_r) * 1e3,
                (t_w - t_re) * 1e3, (time.perf_counter() - t_w) * 1e3))
            if k + 1 < steps:
                up_s = up_next
        barrier()
        el = time.perf_counter() - t0
        if pool:
            pool.shutdown()
        hscene.pin(False)
        if dist:
            tt = torch.tensor([el], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            el = float(tt.item())
        return npix * spp * world * steps / el / 1e6

    e2e_value = e2e_run(hs, "host-built trees", overlap=True)
    e2e_serial = e2e_run(hs, "host-built trees, serial", overlap=False)
    e2e_dev = None
    if not args.no_device_bvh and not args.no_e2e:
        hd = G.HostScene.load_xml(xml, device_blas=True)
        e2e_dev = e2e_run(hd, "trees built at upload", overlap=True)
        hd.close()
    # the other mode on the same scene, for the batched-vs-plain comparison
    other = []
    for k in range(min(2, args.steps)):
        _, st = ctx.render(sid, spp=spp, first_pass=first, batched=not batched, film=film)
        other.append(st["ms"])
    other_value = npix * spp / (sum(other) / len(other) / 1000.0) / 1e6 if other else None

    # lanes busy per warp step in the extend traversal's two phases, with the tuned settings
    # (counting variant, 8 passes)
    _, pst = ctx.render(sid, spp=8, first_pass=first, profile=2, batched=batched)
    simt = {"node_phase": pst["extend_nodes"] / (32.0 * max(1, pst["extend_node_warp_steps"])),
            "leaf_phase": pst["extend_leaf_steps"] / (32.0 * max(1, pst["extend_leaf_warp_steps"])),
            "node_steps_per_leaf_step": pst["extend_node_warp_steps"] / max(1, pst["extend_leaf_warp_steps"]),
            "note": "fraction of a warp's 32 lanes busy per step (node visits or leaf steps / 32 x warp steps), "
                    "counting variant of kExtend, 8 passes with the tuned settings"}

    peaks, peak_kind = measured_peaks()
    bytes_per_ray = nodes_per_ray * 128 + tris_per_ray * 48 + 32 + 32
    ext_launches = iters
    achieved = (bytes_per_ray * ext_rays) / (ext_ms / 1000.0) / 1e9 if ext_ms > 0 else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", "extend_traffic.json")
    if os.path.exists(tp) and ext_launches:
        # DRAM bytes per extend ray from one ncu capture, scaled to this run's average launch
        with open(tp) as f:
            per_ray = json.load(f).get("dram_bytes_per_ray")
        if per_ray:
            traffic = per_ray * ext_rays / ext_launches
    launches_total = sum(s["launches"] for s in stats)
    line = {
        "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * elapsed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator, gianduia_b200/scenes.py)",
        "config": {"workload": "microfacet 1024x1024, 64 spp, path_gpu depth 16, 5,242,882 tris, 4105 instances, 8 sphere lights",
                   "parallelism": "spp-sharded" if world > 1 else "single GPU",
                   "mode": "batched (all passes share a refilled pool of path slots)" if batched else "plain (one pass in flight)",
                   "l2": "inputs larger than L2 (scene %.2f GB resident)" % (scene_bytes / 1e9),
                   "graphs": "per-bounce loop replayed as CUDA graphs" if tune.get("graphs") else "graphs off",
                   "tune": tune},
        "mrays_per_s": rays * world / elapsed / 1e6,
        ("plain_value" if batched else "batched_value"): other_value,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": (achieved / peaks["hbm_gbs"]) if achieved else None, "traffic": traffic,
                     "kernel": "kExtend (closest-hit BVH4 traversal)",
                     "bytes_per_ray": bytes_per_ray, "nodes_per_ray": nodes_per_ray, "tris_per_ray": tris_per_ray,
                     "launches": ext_launches, "ms_total": ext_ms, "lanes_busy": simt,
                     "peak_kind": peak_kind + " (copy bandwidth)",
                     "timed_in": "a separate instrumented render of the same %d passes (CUDA events around each "
                                 "extend launch, graphs off); the headline steps run the CUDA-graph loop" % spp},
        "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": int(scene_bytes),
                "d2h_bytes_per_step": int(film_bytes),
                "note": "every step uploads its own copy of the scene from pinned host memory, renders it "
                        "and reads the film back; the upload of step k + 1 runs on a second host thread "
                        "during step k's render (the first step's upload is not overlapped)",
                "serial_value": e2e_serial},
        "e2e_device_trees": None if e2e_dev is None else {
            "value": e2e_dev, "unit": "Mpaths/s",
            "note": "mesh trees built on the GPU inside each timed upload, overlapped as in e2e"},
        "gpu_launches": int(launches_total),
        "clocks": clk,
    }
    if film_check is not None:
        line["reduced_film"] = film_check
    if rank == 0 and world == 1 and not args.no_traversal:
        line["traversal"] = traversal_leg(ctx)
    if rank == 0 and world == 1 and not args.no_scenes:
        line["scenes"] = scenes_leg(ctx)
        line["microfacet_gaussian"] = gaussian_leg(ctx, hs, tune, spp)
    if rank == 0 and world == 1 and not args.no_device_bvh:
        line["device_bvh"] = device_bvh_leg(ctx, xml, sid, host_load_s, tune)
        line["cold_request"] = cold_request_leg(ctx, xml, spp)
    if rank == 0 and world == 1 and args.serve_requests > 0:
        line["serve"] = serve_leg(ctx, sid, args.serve_requests)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(xml)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.free_scene(sid)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
