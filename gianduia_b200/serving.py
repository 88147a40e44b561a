"""Serving workload: a stream of render requests over three scenes -- the Cornell box
(path_gpu), the microfacet sphere grid (path_gpu) and the volumetric Cornell box
(volpath_gpu) -- with Poisson arrivals, served two ways:

  served : every request is submitted to the context's job server (gnd_gpu_serve_*) at
           its arrival time; jobs share one pool of path slots, oldest job first.
  plain  : one request at a time through gnd_gpu_render (one sample pass in flight),
           first come first served. Its time-to-image follows from each request's
           measured render time by the single-server FIFO recurrence
           finish_i = max(arrival_i, finish_{i-1}) + service_i.

Per request, uniformly: scene, square resolution in {128, 256, 512, 1024}, spp in
{4, 16, 64}, maximum depth in 8..32. Time-to-image runs from arrival to the finished
film in host memory."""
import queue
import threading
import time

import numpy as np

SCENES = ("cornell", "microfacet", "volumetric")
RESOLUTIONS = (128, 256, 512, 1024)
SPPS = (4, 16, 64)
DEPTH_MIN, DEPTH_MAX = 8, 32


def make_requests(n, seed=4):
    """n requests as dicts (scene, res, spp, max_depth), drawn uniformly and seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        out.append(dict(scene=SCENES[int(rng.integers(len(SCENES)))], res=int(RESOLUTIONS[int(rng.integers(4))]),
                        spp=int(SPPS[int(rng.integers(3))]), max_depth=int(rng.integers(DEPTH_MIN, DEPTH_MAX + 1))))
    return out


def mean_samples_per_request():
    """Expected samples (paths) per request: E[res^2] * E[spp]."""
    return float(np.mean([r * r for r in RESOLUTIONS]) * np.mean(SPPS))


def poisson_arrivals(n, rate, seed=4):
    """Arrival times in seconds of a Poisson process of `rate` requests/s (exponential gaps)."""
    if rate <= 0:
        raise ValueError("rate must be positive")
    rng = np.random.default_rng(seed + 1)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def fifo_finish(arrivals, service):
    """Finish times of a single first-come first-served server."""
    arrivals = np.asarray(arrivals, np.float64)
    service = np.asarray(service, np.float64)
    if arrivals.shape != service.shape:
        raise ValueError("arrivals and service times differ in length")
    f = np.empty_like(arrivals)
    t = 0.0
    for i in range(arrivals.shape[0]):
        t = max(t, arrivals[i]) + service[i]
        f[i] = t
    return f


def latency_stats(lat):
    lat = np.asarray(lat, np.float64)
    return dict(p50=float(np.percentile(lat, 50)), p99=float(np.percentile(lat, 99)), mean=float(lat.mean()),
                max=float(lat.max()))


def samples(req):
    return req["res"] * req["res"] * req["spp"]


def run_served(ctx, sids, integrators, reqs, arrivals):
    """Submits request i at arrivals[i] seconds after the start and collects every film.
    Returns (time-to-image per request in s, makespan in s)."""
    n = len(reqs)
    ids = queue.Queue()
    done = [None] * n
    errors = []

    def waiter():
        for _ in range(n):
            i, jid, late_s = ids.get()
            try:
                _, st = ctx.wait(jid)
                done[i] = (st, late_s)
            except Exception as e:   # recorded and re-raised by the caller
                errors.append(e)
                done[i] = None

    th = threading.Thread(target=waiter, daemon=True)
    th.start()
    t0 = time.perf_counter()
    for i, r in enumerate(reqs):
        delay = arrivals[i] - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        late = (time.perf_counter() - t0) - arrivals[i]
        jid = ctx.submit(sids[r["scene"]], width=r["res"], height=r["res"], spp=r["spp"], max_depth=r["max_depth"],
                         integrator=integrators[r["scene"]])
        ids.put((i, jid, late))
    th.join()
    makespan = time.perf_counter() - t0
    if errors:
        raise errors[0]
    # time-to-image = lateness of the submission + (film ready - submitted) on the server clock
    lat = [late + (st["done_ms"] - st["submit_ms"]) * 1e-3 for st, late in done]
    return np.asarray(lat), makespan


def run_plain_service(ctx, sids, integrators, reqs):
    """Host wall time of each request rendered alone with gnd_gpu_render (plain mode)."""
    out = np.empty(len(reqs))
    for i, r in enumerate(reqs):
        t = time.perf_counter()
        ctx.render(sids[r["scene"]], spp=r["spp"], max_depth=r["max_depth"], integrator=integrators[r["scene"]],
                   width=r["res"], height=r["res"])
        out[i] = time.perf_counter() - t
    return out


def calibrate_capacity(ctx, sids, integrators, n=24, seed=40):
    """Requests per second the job server sustains: n requests of the same distribution
    submitted at once, n / makespan, timed on a second submission (the first one warms the
    server up: its path pool, the kernels' first loads and the captured graphs)."""
    reqs = make_requests(n, seed)
    run_served(ctx, sids, integrators, reqs, np.zeros(n))
    _, makespan = run_served(ctx, sids, integrators, reqs, np.zeros(n))
    return n / makespan, sum(samples(r) for r in reqs) / makespan
