"""gnd_gpu_trace_closest_fixed: the allocation-free closest-hit entry point, checked
against gnd_gpu_trace_closest on the same rays (same kernel, so hits are expected
bit-equal), on two calls in a row with different batches, plus its size limit.
Runs alone or after every other test (the file name sorts last)."""
import ctypes

import numpy as np
import pytest

import gianduia_b200 as G
from gianduia_b200 import scenes

pytestmark = pytest.mark.gpu

MAX_RAYS = 65536   # GND_TRACE_FIXED_MAX_RAYS
T_REL = 0.0        # same kernel and arithmetic as gnd_gpu_trace_closest: bit-equal t


def trace_fixed(ctx, sid, rays):
    L = G.lib()
    fn = L.gnd_gpu_trace_closest_fixed
    fn.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
    fn.restype = ctypes.c_int32
    r = G.as_rays(rays)
    hits = np.zeros(r.shape[0], G.HIT_DTYPE)
    status = fn(ctx._h, sid, r.ctypes.data, r.shape[0], hits.ctypes.data)
    return status, hits


def assert_same(a, b, label):
    assert np.array_equal(a["inst"], b["inst"]), label + ": instance differs"
    assert np.array_equal(a["prim"], b["prim"]), label + ": primitive differs"
    h = a["inst"] >= 0
    rel = np.abs(a["t"][h] - b["t"][h]) / np.maximum(np.abs(b["t"][h]), 1e-30)
    assert rel.max(initial=0.0) <= T_REL, label + ": t differs (max rel %g)" % rel.max(initial=0.0)
    assert np.array_equal(a["u"][h], b["u"][h]) and np.array_equal(a["v"][h], b["v"][h]), label + ": barycentrics differ"


def test_fixed_matches_trace_closest():
    ctx = G.GpuContext(0)
    try:
        tris = scenes.random_triangles(1 << 16, seed=7)
        sid = ctx.upload(G.HostScene.from_triangles(tris))
        batches = [scenes.random_rays(MAX_RAYS, seed=11), scenes.random_rays(40000, seed=12)]
        for k, rays in enumerate(batches):
            status, got = trace_fixed(ctx, sid, rays)
            assert status == G.GND_OK, G.lib().gnd_last_error().decode()
            ref = ctx.trace_closest(sid, rays)
            assert (ref["inst"] >= 0).mean() > 0.05, "batch %d: too few hits to compare" % k
            assert_same(got, ref, "call %d" % k)
        # a batch over the limit is rejected with GND_ERR_INVALID and a message naming it
        status, _ = trace_fixed(ctx, sid, scenes.random_rays(MAX_RAYS + 1, seed=13))
        assert status == 1   # GND_ERR_INVALID
        assert b"65536" in G.lib().gnd_last_error()
        # an empty batch is a no-op
        status, got = trace_fixed(ctx, sid, scenes.random_rays(0, seed=14))
        assert status == G.GND_OK and got.shape[0] == 0
    finally:
        ctx.close()
