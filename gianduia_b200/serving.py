"""Serving workload: a stream of render requests over three scenes -- the Cornell box
(path_gpu), the microfacet sphere grid (path_gpu) and the volumetric Cornell box
(volpath_gpu) -- with Poisson arrivals, served two ways:

  served : every request is submitted to the context's job server (gnd_gpu_serve_*) at
           its arrival time; jobs share one pool of path slots, oldest job first.
  plain  : one request at a time through gnd_gpu_render (one sample pass in flight),
           first come first served. Its time-to-image follows from each request's
           render time by the single-server FIFO recurrence
           finish_i = max(arrival_i, finish_{i-1}) + service_i. The render time is
           measured per request (run_plain_service) or, for long streams, modelled from
           measured renders (plain_service_model): a plain render runs its passes one
           after another, so its time is a fixed part plus spp times a per-pass part,
           both measured for every (scene, resolution, depth) of the stream.

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


def _plain_time(ctx, sid, integrator, res, spp, depth):
    t = time.perf_counter()
    ctx.render(sid, spp=spp, max_depth=depth, integrator=integrator, width=res, height=res)
    return time.perf_counter() - t


def plain_service_model(ctx, sids, integrators, reqs, check=6):
    """Plain (one pass in flight) render times of the requests without rendering each one:
    for every distinct (scene, resolution, depth) of the stream a 1-pass and a 4-pass
    plain render are timed (host wall time, as run_plain_service), giving
    time(spp) = fixed + spp * per_pass with per_pass = (t4 - t1) / 3. `check` requests of
    spp 16 or 64 are also rendered in full and compared with the model.
    Returns (service times in s, dict with the model's size and its largest relative error)."""
    keys = sorted({(r["scene"], r["res"], r["max_depth"]) for r in reqs})
    model = {}
    for sc, res, depth in keys:
        sid, integ = sids[sc], integrators[sc]
        _plain_time(ctx, sid, integ, res, 1, depth)   # warm-up (first use of this film size)
        t1 = _plain_time(ctx, sid, integ, res, 1, depth)
        t4 = _plain_time(ctx, sid, integ, res, 4, depth)
        per = max((t4 - t1) / 3.0, 0.0)
        model[(sc, res, depth)] = (max(t1 - per, 0.0), per)

    def predict(r):
        fixed, per = model[(r["scene"], r["res"], r["max_depth"])]
        return fixed + r["spp"] * per

    svc = np.array([predict(r) for r in reqs])
    errs = []
    big = [r for r in reqs if r["spp"] >= 16][:check]
    for r in big:
        meas = _plain_time(ctx, sids[r["scene"]], integrators[r["scene"]], r["res"], r["spp"], r["max_depth"])
        errs.append(abs(predict(r) - meas) / meas)
    return svc, {"keys": len(keys), "checked": len(errs), "max_rel_err": float(max(errs)) if errs else None}


def calibrate_capacity(ctx, sids, integrators, n=200, warm=24, seed=40):
    """What the job server sustains when saturated: n requests of the stream's
    distribution submitted at once, timed from the first submission to the last film
    (after a warm-up submission of `warm` others: the server's path pool, the kernels'
    first loads and the captured graphs). Returns (requests/s, samples/s)."""
    run_served(ctx, sids, integrators, make_requests(warm, seed + 1), np.zeros(warm))
    reqs = make_requests(n, seed)
    _, makespan = run_served(ctx, sids, integrators, reqs, np.zeros(n))
    return n / makespan, sum(samples(r) for r in reqs) / makespan
