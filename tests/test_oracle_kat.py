"""Pins the CPU oracle to the known-answer values and statistical checks in the
reference's own unit tests (tests/**/*_test.cpp of daverlez/gianduia). Every number
asserted here is the one the cited reference test asserts."""
import math

import numpy as np
import pytest

from oracle import pyoracle as O

FLT_EQ = 4 * np.finfo(np.float32).eps  # gtest EXPECT_FLOAT_EQ is 4 ULPs


def feq(a, b):
    a = np.float32(a); b = np.float32(b)
    if a == b:
        return True
    return abs(float(a) - float(b)) <= 4 * np.spacing(np.float32(max(abs(a), abs(b))))


# ---------------------------------------------------------------- fresnel_test.cpp
def test_fr_dielectric():  # fresnel_test.cpp:6-16
    assert feq(O.fr_dielectric(1.0, 1.0, 1.5), 0.04)
    assert feq(O.fr_dielectric(-1.0, 1.0, 1.5), 0.04)
    assert abs(O.fr_dielectric(0.0, 1.0, 1.5) - 1.0) < 1e-6
    assert feq(O.fr_dielectric(-0.5, 1.0, 1.5), 1.0)


def test_refract():  # fresnel_test.cpp:18-47
    ok, wt = O.refract((0, 0, -1), (0, 0, 1), 1.5)
    assert ok and feq(wt[0], 0) and feq(wt[1], 0) and feq(wt[2], -1)
    wi = np.array([1, 0, -1], np.float32) / np.float32(math.sqrt(2))
    ok, wt = O.refract(wi, (0, 0, 1), 1.0 / 1.5)
    assert ok
    assert abs(np.linalg.norm(wt) - 1) < 1e-5
    assert abs(abs(wt[0]) - (1.0 / 1.5) * wi[0]) < 1e-5
    wi_in = np.array([1, 0, 1], np.float32) / np.float32(math.sqrt(2))
    ok, _ = O.refract(wi_in, (0, 0, -1), 1.5)
    assert not ok


def test_fr_conductor():  # fresnel_test.cpp:49-65
    r = O.fr_conductor(1.0, (1, 1, 1), (1.5, 1.5, 1.5), (2, 2, 2))
    assert np.all(np.abs(r - 0.414634) < 1e-5)
    g = O.fr_conductor(0.0, (1, 1, 1), (1.5, 1.5, 1.5), (2, 2, 2))
    assert all(feq(x, 1.0) for x in g)


# ---------------------------------------------------------------- transmission_test.cpp
def test_specular_transmission():  # transmission_test.cpp:6-52
    p = O.lobe_params(T=(0.9, 0.9, 0.9), eta_ext=1.0, eta_int=1.5)
    f, pdf = O.bxdf_eval(7, p, (0, 0, 1), (0, 0, -1))
    assert f[0] == 0 and pdf == 0
    wi, w, pdf, typ = O.bxdf_sample(7, p, (0, 0, 1), (0.5, 0.5), 0.5)
    assert feq(wi[0], 0) and feq(wi[1], 0) and feq(wi[2], -1)
    assert feq(pdf, 1.0)
    assert typ & 2 and typ & 16
    F = O.fr_dielectric(1.0, 1.0, 1.5)
    r = np.float32(1.0) / np.float32(1.5)
    assert feq(w[0], np.float32(0.9) * (np.float32(1) - np.float32(F)) * (r * r))
    wi, w, pdf, typ = O.bxdf_sample(7, p, (0, 0, -1), (0.5, 0.5), 0.5)
    assert feq(wi[2], 1.0)
    r = np.float32(1.5) / np.float32(1.0)
    assert feq(w[0], np.float32(0.9) * (np.float32(1) - np.float32(F)) * (r * r))
    wo = np.array([1, 0, -0.1], np.float32); wo /= np.linalg.norm(wo)
    _, w, _, _ = O.bxdf_sample(7, p, wo, (0.5, 0.5), 0.5)
    assert np.all(w == 0)


# ---------------------------------------------------------------- microfacet_test.cpp
def test_roughness_to_alpha():  # microfacet_test.cpp:6-12
    assert feq(O.roughness_to_alpha(0.5), 0.25)
    assert feq(O.roughness_to_alpha(1.0), 1.0)
    assert feq(O.roughness_to_alpha(0.0), 1e-6)
    assert feq(O.roughness_to_alpha(1e-5), 1e-6)


def test_ggx_d_g():  # microfacet_test.cpp:14-33
    assert feq(O.ggx(0, 0.5, (0, 0, 1)), 4.0 * 0.31830988618379067154)
    assert feq(O.ggx(1, 0.5, (0, 0, 1)), 1.0)
    assert feq(O.ggx(2, 0.5, (0, 0, 1), (0, 0, 1)), 1.0)
    g = np.array([1, 0, 0.01], np.float32); g /= np.linalg.norm(g)
    assert O.ggx(1, 0.5, g) < 0.1


def test_ggx_sampling_pdf():  # microfacet_test.cpp:35-50
    wo = np.array([1, 1, 1], np.float32); wo /= np.linalg.norm(wo)
    wh = O.ggx(4, 0.5, wo, (0.3, 0.7))
    assert abs(np.linalg.norm(wh) - 1) < 1e-5
    assert wh[2] * wo[2] >= 0
    pdf = O.ggx(3, 0.5, wo, wh)
    exp = np.float32(O.ggx(0, 0.5, wh)) * np.float32(O.ggx(1, 0.5, wo)) * np.float32(abs(np.dot(wo, wh))) / np.float32(abs(wo[2]))
    assert abs(pdf - exp) <= 1e-5 * abs(exp)


# ---------------------------------------------------------------- reflection_test.cpp
def test_lambertian():  # reflection_test.cpp:7-24
    p = O.lobe_params(R=(0.9, 0.1, 0.1))
    wi = np.array([1, 1, 1], np.float32); wi /= np.linalg.norm(wi)
    f, pdf = O.bxdf_eval(0, p, (0, 0, 1), wi)
    inv_pi = np.float32(0.31830988618379067154)
    assert feq(f[0], np.float32(0.9) * inv_pi) and feq(f[1], np.float32(0.1) * inv_pi)
    assert feq(pdf, max(0.0, wi[2] * inv_pi))
    _, pdf = O.bxdf_eval(0, p, (0, 0, 1), (0, 0, -1))
    assert pdf == 0


def test_specular_reflection():  # reflection_test.cpp:26-52
    p = O.lobe_params(R=(0.8, 0.8, 0.8))
    wo = np.array([1, 0, 1], np.float32); wo /= np.linalg.norm(wo)
    f, pdf = O.bxdf_eval(1, p, wo, (0, 0, 1))
    assert f[0] == 0 and pdf == 0
    wi, w, pdf, typ = O.bxdf_sample(1, p, wo, (0.5, 0.5), 0.5)
    assert feq(wi[0], -wo[0]) and feq(wi[1], -wo[1]) and feq(wi[2], wo[2])
    assert feq(pdf, 1.0) and typ & 1 and typ & 16


def test_fresnel_specular():  # reflection_test.cpp:54-74
    p = O.lobe_params(R=(1, 1, 1), T=(1, 1, 1), eta_ext=1.0, eta_int=1.5)
    wo = np.array([1, 0, 1], np.float32); wo /= np.linalg.norm(wo)
    wi, _, _, typ = O.bxdf_sample(2, p, wo, (0.0, 0.5), 0.5)
    assert feq(wi[0], -wo[0]) and feq(wi[2], wo[2])
    assert typ & 1 and typ & 16
    f, pdf = O.bxdf_eval(2, p, wo, wi)
    assert f[0] == 0 and pdf == 0


def test_microfacet_reflection():  # reflection_test.cpp:76-112
    p = O.lobe_params(R=(0.8, 0.8, 0.8), alpha=0.5)
    wo = np.array([1, 0, 1], np.float32); wo /= np.linalg.norm(wo)
    wi = np.array([-1, 0, 1], np.float32); wi /= np.linalg.norm(wi)
    ff, _ = O.bxdf_eval(3, p, wo, wi)
    fb, _ = O.bxdf_eval(3, p, wi, wo)
    assert feq(ff[0], fb[0]) and ff[0] > 0
    ws, w, pdf, typ = O.bxdf_sample(3, p, wo, (0.1, 0.1), 0.5)
    if pdf > 0:
        assert ws[2] * wo[2] > 0 and typ & 8 and typ & 1
        ef, ep = O.bxdf_eval(3, p, wo, ws)
        assert feq(pdf, ep) and feq(w[0], ef[0])


def test_microfacet_fresnel():  # reflection_test.cpp:114-138
    p = O.lobe_params(R=(0.8, 0.8, 0.8), T=(0.8, 0.8, 0.8), eta_ext=1.0, eta_int=1.5, alpha=0.5)
    wo = np.array([1, 0, 1], np.float32); wo /= np.linalg.norm(wo)
    ws, _, pdf, typ = O.bxdf_sample(4, p, wo, (0.1, 0.1), 0.01)
    if pdf > 0:
        assert typ & 8 and typ & 1
        assert feq(pdf, O.bxdf_eval(4, p, wo, ws)[1])
    ws, _, pdf, typ = O.bxdf_sample(4, p, wo, (0.1, 0.1), 0.99)
    if pdf > 0:
        assert typ & 8 and typ & 2
        assert feq(pdf, O.bxdf_eval(4, p, wo, ws)[1])


def test_smooth_plastic():  # reflection_test.cpp:140-163
    p = O.lobe_params(R=(0.5, 0.5, 0.5), T=(0.5, 0.5, 0.5), eta_int=1.5)
    wo = (0, 0, 1)
    wi = np.array([1, 0, 1], np.float32); wi /= np.linalg.norm(wi)
    Fo = np.float32(O.fr_dielectric(1.0, 1.0, 1.5)); Fi = np.float32(O.fr_dielectric(float(wi[2]), 1.0, 1.5))
    exp = np.float32(0.5) * np.float32(0.31830988618379067154) * (np.float32(1) - Fo) * (np.float32(1) - Fi)
    f, _ = O.bxdf_eval(5, p, wo, wi)
    assert feq(f[0], exp)
    ws, _, _, typ = O.bxdf_sample(5, p, wo, (0.5, 0.5), 0.01)
    assert typ & 16 and feq(ws[0], 0)
    _, _, _, typ = O.bxdf_sample(5, p, wo, (0.5, 0.5), 0.99)
    assert typ & 4


def test_rough_plastic():  # reflection_test.cpp:165-188
    p = O.lobe_params(R=(0.5, 0.5, 0.5), T=(0.5, 0.5, 0.5), eta_int=1.5, alpha=0.5)
    wo = np.array([1, 0, 1], np.float32); wo /= np.linalg.norm(wo)
    ws, _, pdf, typ = O.bxdf_sample(6, p, wo, (0.2, 0.2), 0.01)
    if pdf > 0:
        assert typ & 8 and typ & 1
        assert feq(pdf, O.bxdf_eval(6, p, wo, ws)[1])
    ws, _, pdf, typ = O.bxdf_sample(6, p, wo, (0.5, 0.5), 0.99)
    if pdf > 0:
        assert typ & 4 and typ & 1
        assert feq(pdf, O.bxdf_eval(6, p, wo, ws)[1])


# ---------------------------------------------------------------- warp_test.cpp
def _chi2(samples_fn, binner):
    # warp_test.cpp:8-33: PCG32(42), 20x20 bins, 1e5 samples, threshold 600
    draws = O.pcg32(42, 1, 200000).astype(np.float64)
    u = (np.ldexp(draws.astype(np.float32), -32)).astype(np.float32).reshape(-1, 2)
    obs = np.zeros(400, np.int64)
    for k in range(u.shape[0]):
        bx, by = binner(samples_fn(u[k]))
        if 0 <= bx < 20 and 0 <= by < 20:
            obs[by * 20 + bx] += 1
    exp = u.shape[0] / 400.0
    return float(np.sum((obs - exp) ** 2 / exp))


def _phi(x, y):
    p = math.atan2(y, x)
    return p + 2 * math.pi if p < 0 else p


@pytest.mark.parametrize("op,binner", [
    (0, lambda p: (min(int((p[0] ** 2 + p[1] ** 2) * 20), 19), min(int(_phi(p[0], p[1]) / (2 * math.pi) * 20), 19))),
    (1, lambda v: (min(int((v[2] + 1) * 0.5 * 20), 19), min(int(_phi(v[0], v[1]) / (2 * math.pi) * 20), 19))),
    (2, lambda v: (min(int(v[2] * 20), 19), min(int(_phi(v[0], v[1]) / (2 * math.pi) * 20), 19))),
    (3, lambda v: (min(int(v[2] * v[2] * 20), 19), min(int(_phi(v[0], v[1]) / (2 * math.pi) * 20), 19))),
])
def test_warp_chi2(op, binner):  # warp_test.cpp:35-89
    assert _chi2(lambda u: O.warp(op, u), binner) < 600.0


# ---------------------------------------------------------------- frame_test.cpp
def test_frame():  # frame_test.cpp:17-67
    n = np.array([1, 2, 3], np.float32); n /= np.linalg.norm(n)
    f = O.frame(n)
    assert all(feq(f[2][i], n[i]) for i in range(3))
    assert abs(np.linalg.norm(f[0]) - 1) < 1e-6 and abs(np.linalg.norm(f[1]) - 1) < 1e-6
    assert abs(np.dot(f[0], f[1])) < 1e-6 and abs(np.dot(f[0], f[2])) < 1e-6 and abs(np.dot(f[1], f[2])) < 1e-6
    f = O.frame((0, 1, 0))
    w = np.array([1, 1, 0], np.float32); w /= np.linalg.norm(w)
    loc = np.array([w @ f[0], w @ f[1], w @ f[2]])
    back = f[0] * loc[0] + f[1] * loc[1] + f[2] * loc[2]
    assert np.all(np.abs(back - w) < 1e-6)


# ---------------------------------------------------------------- shapes, bounds, camera
def test_sphere():  # sphere_test.cpp:28-84
    out = O.shape_hit(0, (2.0,), (0, 0, 5, 1e-4, 0, 0, -1, np.inf))
    assert out[0] == 1 and feq(out[1], 3) and feq(out[4], 2) and feq(out[7], 1)
    assert feq(out[2], 0) and feq(out[3], 0) and feq(out[5], 0) and feq(out[6], 0)
    out = O.shape_hit(0, (1.0,), (5, 0, 0, 1e-4, 0, 1, 0, np.inf))
    assert out[0] == 0
    out = O.shape_hit(0, (2.0,), (5, 0, 0, 1e-4, 0, 1, 0, np.inf))
    assert feq(out[8], np.float32(0.07957747154594766788) / np.float32(4.0))


def test_cube():  # cube_test.cpp:27-76
    out = O.shape_hit(1, (1, 1, 1), (5, 0, 0, 1e-4, -1, 0, 0, np.inf))
    assert out[0] == 1 and feq(out[1], 4) and feq(out[2], 1) and feq(out[5], 1)
    assert feq(out[3], 0) and feq(out[4], 0) and feq(out[6], 0) and feq(out[7], 0)
    out = O.shape_hit(1, (1, 1, 1), (5, 5, 0, 1e-4, -1, 0, 0, np.inf))
    assert out[0] == 0
    out = O.shape_hit(1, (1, 2, 3), (5, 5, 0, 1e-4, -1, 0, 0, np.inf))
    assert feq(out[8], 1.0 / (2.0 * (2 * 4 + 2 * 6 + 4 * 6)))


def test_bounds_slab():  # bounds_test.cpp:50-69
    h, t = O.bounds_hit((-1, -1, -1), (1, 1, 1), (-3, 0, 0, 1e-4, 1, 0, 0, np.inf))
    assert h and feq(t[0], 2) and feq(t[1], 4)
    h, _ = O.bounds_hit((-1, -1, -1), (1, 1, 1), (-3, 2, 0, 1e-4, 1, 0, 0, np.inf))
    assert not h
    h, t = O.bounds_hit((-1, -1, -1), (1, 1, 1), (0, 0, 0, 1e-4, 0, 1, 0, np.inf))
    assert h and feq(t[0], 0) and feq(t[1], 1)
    h, _ = O.bounds_hit((-1, -1, -1), (1, 1, 1), (-3, 0, 0, 1e-4, 1, 0, 0, 1.0))
    assert not h


def test_perspective():  # perspective_test.cpp:18-61
    o, d = O.perspective(60.0, 1280, 720, 0.5, 0.5)
    assert all(feq(x, 0) for x in o) and feq(d[0], 0) and feq(d[1], 0) and feq(d[2], -1)
    _, d = O.perspective(90.0, 800, 800, 1.0, 1.0)
    s = 1 / math.sqrt(3)
    assert abs(d[0] - s) < 1e-5 and abs(d[1] - s) < 1e-5 and abs(d[2] + s) < 1e-5


# ---------------------------------------------------------------- sampler stream (pcg32.h / independent.cpp)
def test_pcg32_reference_stream():
    # The PCG32 XSH-RR generator (pcg32.h:5-32) reproduces the published pcg32 demo
    # stream for seed (42, 54): the first six outputs printed by pcg32-demo.
    out = O.pcg32(42, 54, 6)
    assert list(out) == [0xa15c02b7, 0x7b47f409, 0xba1d3330, 0x83d2f293, 0xbfa4784b, 0xcbed606e]


def test_sampler_seeding_matches_python_restatement():
    # independent.cpp:22-32 + pcg32.h: restated in numpy integer arithmetic as a check.
    M = (1 << 64) - 1

    def smix(x):
        z = (x + 0x9e3779b97f4a7c15) & M
        z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & M
        z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & M
        return z ^ (z >> 31)

    def pcg(state, inc):
        old = state
        state = (old * 6364136223846793005 + inc) & M
        xs = (((old >> 18) ^ old) >> 27) & 0xffffffff
        rot = old >> 59
        return state, ((xs >> rot) | (xs << ((-rot) & 31))) & 0xffffffff

    for key in (0, 1, 12345, 65535 + 7 * 65536):
        assert O.splitmix64(key) == smix(key)
        inc = (1 << 1) | 1
        st, _ = pcg(0, inc)
        st = (st + smix(key)) & M
        st, _ = pcg(st, inc)
        vals = []
        for _ in range(8):
            st, r = pcg(st, inc)
            vals.append(np.ldexp(np.float32(r), -32).astype(np.float32))
        got = O.sampler_floats(key, 8)
        assert np.array_equal(np.array(vals, np.float32), got)


# ---------------------------------------------------------------- homogeneous medium, HG (restated; no reference test)
def test_medium_sample_weights():
    # homogeneous.cpp:32-63: a surface hit before the sampled distance returns Tr/mean(Tr)
    w = O.medium_sample((0.1, 0.1, 0.1), (0.1, 0.1, 0.1), 0.5, 0.2, 0.999999, (0, 0, 1))
    assert w[3] == 0 and abs(w[0] - 1.0) < 1e-6
    w = O.medium_sample((0.05, 0.05, 0.05), (0.5, 0.5, 0.5), 100.0, 0.2, 0.5, (0, 0, 1))
    sig_t = 0.55
    assert w[3] == 1 and abs(w[4] - (-math.log(0.5) / sig_t)) < 1e-5
    assert abs(w[0] - 1.0 / sig_t) < 1e-5


def test_hg_normalised():
    # the HG value (phase.h:84-87) integrates to one over the sphere
    g = 0.6
    n = 200000
    rng = np.random.default_rng(3)
    z = rng.uniform(-1, 1, n)
    vals = np.array([O.hg(0, g, (0, 0, 1), (math.sqrt(max(0, 1 - zz * zz)), 0, zz)) for zz in z[:2000]])
    assert abs(vals.mean() * 4 * math.pi - 1.0) < 0.05
