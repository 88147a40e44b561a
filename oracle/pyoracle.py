"""Oracle (test infrastructure only): ctypes bindings of the CPU restatement of the
reference's radiance path (oracle/src). Imported by tests/, the smoke check and the
bench's CPU-baseline leg, never by the product package.
"""
import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None
_lock = threading.Lock()

_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def build():
    """Compiles oracle/_build/liboracle.so with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(_LIB_PATH)
            L.orc_load_scene.restype = ctypes.c_void_p
            L.orc_load_scene.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
            L.orc_mesh_scene.restype = ctypes.c_void_p
            L.orc_mesh_scene.argtypes = [_f32p, ctypes.c_int64, ctypes.c_char_p, ctypes.c_int]
            L.orc_free_scene.argtypes = [ctypes.c_void_p]
            L.orc_scene_info.argtypes = [ctypes.c_void_p, _i32p]
            L.orc_render.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 7 + [_f32p, _u64p, ctypes.c_char_p, ctypes.c_int]
            L.orc_render_fixed.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 7 + [_u64p, _f32p, _u64p, ctypes.c_char_p,
                                                                                   ctypes.c_int]
            L.orc_trace.argtypes = [ctypes.c_void_p, _f32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                    _f32p, _f32p, _f32p, _i32p, _i32p, _u32p, _u32p]
            L.orc_trace_interaction.argtypes = [ctypes.c_void_p, _f32p, ctypes.c_int64, ctypes.c_int, _f32p, _i32p]
            L.orc_camera_rays.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, _i32p, _i32p, _f32p]
            L.orc_fr_dielectric.restype = ctypes.c_float
            L.orc_fr_dielectric.argtypes = [ctypes.c_float] * 3
            L.orc_fr_conductor.argtypes = [ctypes.c_float, _f32p, _f32p, _f32p, _f32p]
            L.orc_refract.argtypes = [_f32p, _f32p, ctypes.c_float, _f32p]
            L.orc_roughness_to_alpha.restype = ctypes.c_float
            L.orc_roughness_to_alpha.argtypes = [ctypes.c_float]
            L.orc_ggx.restype = ctypes.c_float
            L.orc_ggx.argtypes = [ctypes.c_int, ctypes.c_float, _f32p, _f32p, _f32p]
            L.orc_bxdf_eval.argtypes = [ctypes.c_int, _f32p, _f32p, _f32p, _f32p, _f32p]
            L.orc_bxdf_sample.argtypes = [ctypes.c_int, _f32p, _f32p, _f32p, ctypes.c_float, _f32p, _f32p, _f32p, _i32p]
            L.orc_warp.argtypes = [ctypes.c_int, _f32p, _f32p]
            L.orc_pcg32.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _u32p]
            L.orc_splitmix64.restype = ctypes.c_uint64
            L.orc_splitmix64.argtypes = [ctypes.c_uint64]
            L.orc_sampler_floats.argtypes = [ctypes.c_uint64, ctypes.c_int, _f32p]
            L.orc_frame.argtypes = [_f32p, _f32p]
            L.orc_shape_hit.argtypes = [ctypes.c_int, _f32p, _f32p, _f32p]
            L.orc_bounds_hit.argtypes = [_f32p, _f32p, _f32p, _f32p]
            L.orc_perspective.argtypes = [ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, _f32p]
            L.orc_medium_sample.argtypes = [_f32p, _f32p]
            L.orc_hg.restype = ctypes.c_float
            L.orc_hg.argtypes = [ctypes.c_int, ctypes.c_float, _f32p, _f32p, _f32p]
            L.orc_post.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                   ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                   _f32p, ctypes.c_void_p]
            L.orc_env_load.restype = ctypes.c_void_p
            L.orc_env_load.argtypes = [ctypes.c_char_p, ctypes.c_float]
            L.orc_env_free.argtypes = [ctypes.c_void_p]
            L.orc_env_sample.argtypes = [ctypes.c_void_p, ctypes.c_int, _f32p, _f32p, _f32p, _f32p]
            L.orc_env_pdf.argtypes = [ctypes.c_void_p, ctypes.c_int, _f32p, _f32p]
            L.orc_env_eval.argtypes = [ctypes.c_void_p, ctypes.c_int, _f32p, _f32p]
            L.orc_motion_interpolate.argtypes = [_f32p, _f32p, ctypes.c_float, _f32p, _f32p]
            L.orc_round_half.restype = ctypes.c_float
            L.orc_round_half.argtypes = [ctypes.c_float]
            L.orc_perlin_perm.argtypes = [ctypes.POINTER(ctypes.c_int32)]
            L.orc_tex_eval.argtypes = [ctypes.c_char_p, ctypes.c_int64, _f32p, _f32p, ctypes.c_char_p, ctypes.c_int]
            _lib = L
    return _lib


def _fp(a):
    return a.ctypes.data_as(_f32p)


def f32(*v):
    return np.ascontiguousarray(np.array(v, dtype=np.float32).ravel())


class Scene:
    """A scene loaded by the oracle's restatement of the reference loader."""

    def __init__(self, handle):
        self.h = handle
        info = np.zeros(7, np.int32)
        lib().orc_scene_info(self.h, info.ctypes.data_as(_i32p))
        (self.width, self.height, self.spp, self.max_depth, self.kind,
         self.num_primitives, self.num_emitters) = [int(x) for x in info]

    @staticmethod
    def load(xml_path):
        err = ctypes.create_string_buffer(1024)
        h = lib().orc_load_scene(os.fsencode(xml_path), err, 1024)
        if not h:
            raise RuntimeError(err.value.decode())
        return Scene(h)

    @staticmethod
    def from_triangles(tris):
        tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
        err = ctypes.create_string_buffer(1024)
        h = lib().orc_mesh_scene(_fp(tris), tris.shape[0], err, 1024)
        if not h:
            raise RuntimeError(err.value.decode())
        return Scene(h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_free_scene(self.h)
            self.h = None

    def render(self, s0=0, s1=None, window=None, nthreads=0, film=None):
        """Passes [s0, s1) over window (x0, y0, x1, y1); returns (film[H,W,7], paths, rays)."""
        s1 = self.spp if s1 is None else s1
        x0, y0, x1, y1 = window if window else (0, 0, self.width, self.height)
        if film is None:
            film = np.zeros((self.height, self.width, 7), np.float32)
        stats = np.zeros(2, np.uint64)
        err = ctypes.create_string_buffer(1024)
        rc = lib().orc_render(self.h, s0, s1, x0, y0, x1, y1, nthreads, _fp(film),
                              stats.ctypes.data_as(_u64p), err, 1024)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return film, int(stats[0]), int(stats[1])

    def render_fixed(self, s0=0, s1=None, window=None, nthreads=0, fsum=None, fsq=None):
        """As render with the film in fixed point: returns (fsum uint64 [H, W, 4] -- sum wL
        rgb and sum w in units of 2^-24 --, fsq float32 [H, W, 3] -- sum wL^2 --, paths, rays),
        accumulated on top of fsum / fsq when given."""
        s1 = self.spp if s1 is None else s1
        x0, y0, x1, y1 = window if window else (0, 0, self.width, self.height)
        if fsum is None:
            fsum = np.zeros((self.height, self.width, 4), np.uint64)
        if fsq is None:
            fsq = np.zeros((self.height, self.width, 3), np.float32)
        assert fsum.dtype == np.uint64 and fsum.flags.c_contiguous and fsq.dtype == np.float32 and fsq.flags.c_contiguous
        stats = np.zeros(2, np.uint64)
        err = ctypes.create_string_buffer(1024)
        rc = lib().orc_render_fixed(self.h, s0, s1, x0, y0, x1, y1, nthreads, fsum.ctypes.data_as(_u64p), _fp(fsq),
                                    stats.ctypes.data_as(_u64p), err, 1024)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return fsum, fsq, int(stats[0]), int(stats[1])

    def trace(self, rays, anyhit=False, nthreads=0, counters=False):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        t = np.zeros(n, np.float32); u = np.zeros(n, np.float32); v = np.zeros(n, np.float32)
        prim = np.zeros(n, np.int32); inst = np.zeros(n, np.int32)
        nodes = np.zeros(n, np.uint32) if counters else None
        tris = np.zeros(n, np.uint32) if counters else None
        lib().orc_trace(self.h, _fp(rays), n, 1 if anyhit else 0, nthreads, _fp(t), _fp(u), _fp(v),
                        prim.ctypes.data_as(_i32p), inst.ctypes.data_as(_i32p),
                        nodes.ctypes.data_as(_u32p) if counters else None,
                        tris.ctypes.data_as(_u32p) if counters else None)
        if anyhit:
            return inst.astype(bool), nodes, tris
        return dict(t=t, u=u, v=v, prim=prim, inst=inst, nodes=nodes, tris=tris)

    def interactions(self, rays, nthreads=0):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        out = np.zeros((n, 11), np.float32)
        inst = np.zeros(n, np.int32)
        lib().orc_trace_interaction(self.h, _fp(rays), n, nthreads, _fp(out), inst.ctypes.data_as(_i32p))
        return out, inst

    def camera_rays(self, spass, px, py):
        px = np.ascontiguousarray(px, np.int32); py = np.ascontiguousarray(py, np.int32)
        out = np.zeros((px.size, 8), np.float32)
        lib().orc_camera_rays(self.h, spass, px.size, px.ctypes.data_as(_i32p), py.ctypes.data_as(_i32p), _fp(out))
        return out


# ------------------------------------------------------------------ known-answer helpers
def fr_dielectric(c, ext, inn):
    return float(lib().orc_fr_dielectric(c, ext, inn))


def fr_conductor(c, eta_i, eta_t, k):
    out = np.zeros(3, np.float32)
    lib().orc_fr_conductor(c, _fp(f32(eta_i)), _fp(f32(eta_t)), _fp(f32(k)), _fp(out))
    return out


def refract(wi, n, eta):
    out = np.zeros(3, np.float32)
    ok = lib().orc_refract(_fp(f32(wi)), _fp(f32(n)), eta, _fp(out))
    return bool(ok), out


def roughness_to_alpha(r):
    return float(lib().orc_roughness_to_alpha(r))


def ggx(op, alpha, w, w2=None):
    out = np.zeros(3, np.float32)
    w2a = f32(w2) if w2 is not None else None
    v = lib().orc_ggx(op, alpha, _fp(f32(w)), _fp(w2a) if w2a is not None else None, _fp(out))
    return out if op == 4 else float(v)


def lobe_params(R=(0, 0, 0), T=(0, 0, 0), eta_ext=1.0, eta_int=1.5, alpha=0.5, cond_eta=(1, 1, 1), cond_k=(1, 1, 1)):
    return f32(*R, *T, eta_ext, eta_int, alpha, *cond_eta, *cond_k, 0)


def bxdf_eval(kind, params, wo, wi):
    f = np.zeros(3, np.float32); pdf = np.zeros(1, np.float32)
    lib().orc_bxdf_eval(kind, _fp(params), _fp(f32(wo)), _fp(f32(wi)), _fp(f), _fp(pdf))
    return f, float(pdf[0])


def bxdf_sample(kind, params, wo, u, uc):
    wi = np.zeros(3, np.float32); f = np.zeros(3, np.float32); pdf = np.zeros(1, np.float32)
    typ = np.zeros(1, np.int32)
    lib().orc_bxdf_sample(kind, _fp(params), _fp(f32(wo)), _fp(f32(u)), uc, _fp(wi), _fp(f), _fp(pdf),
                          typ.ctypes.data_as(_i32p))
    return wi, f, float(pdf[0]), int(typ[0])


def warp(op, u):
    out = np.zeros(3, np.float32)
    lib().orc_warp(op, _fp(f32(u)), _fp(out))
    return out


def pcg32(initstate, initseq, n):
    out = np.zeros(n, np.uint32)
    lib().orc_pcg32(initstate, initseq, n, out.ctypes.data_as(_u32p))
    return out


def splitmix64(x):
    return int(lib().orc_splitmix64(x))


def sampler_floats(key, n):
    out = np.zeros(n, np.float32)
    lib().orc_sampler_floats(key, n, _fp(out))
    return out


def frame(n):
    out = np.zeros(9, np.float32)
    lib().orc_frame(_fp(f32(n)), _fp(out))
    return out.reshape(3, 3)


def shape_hit(shape, params, ray):
    out = np.zeros(9, np.float32)
    lib().orc_shape_hit(shape, _fp(f32(params)), _fp(f32(ray)), _fp(out))
    return out


def bounds_hit(lo, hi, ray):
    out = np.zeros(2, np.float32)
    h = lib().orc_bounds_hit(_fp(f32(lo)), _fp(f32(hi)), _fp(f32(ray)), _fp(out))
    return bool(h), out


def perspective(fov, w, h, fx, fy):
    out = np.zeros(6, np.float32)
    lib().orc_perspective(fov, w, h, fx, fy, _fp(out))
    return out[:3], out[3:]


def medium_sample(sigma_a, sigma_s, tmax, u0, u1, d):
    out = np.zeros(5, np.float32)
    lib().orc_medium_sample(_fp(f32(*sigma_a, *sigma_s, tmax, u0, u1, *d)), _fp(out))
    return out


def hg(op, g, wo, x):
    out = np.zeros(3, np.float32)
    v = lib().orc_hg(op, g, _fp(f32(wo)), _fp(f32(x)), _fp(out))
    return (float(v), out) if op == 1 else float(v)


# ------------------------------------------------------------------ post-processing
def post(rgb, tonemapper=0, exposure=0.0, bloom=False, threshold=1.0, radius=1.0, intensity=0.04, mips=6, output=0):
    """Post-processing of a linear image [h, w, 3] (tonemap.frag, bloom_*.frag,
    gammaCorrect.frag, Film::savePNG): returns (tonemapped float image, 8-bit image)."""
    rgb = np.ascontiguousarray(rgb, dtype=np.float32)
    h, w = rgb.shape[:2]
    hdr = np.zeros((h, w, 3), np.float32)
    out8 = np.zeros((h, w, 3), np.uint8)
    lib().orc_post(_fp(rgb), w, h, tonemapper, exposure, 1 if bloom else 0, threshold, radius, intensity, mips, output,
                   _fp(hdr), out8.ctypes.data)
    return hdr, out8


def round_half(x):
    return float(lib().orc_round_half(x))


class EnvMap:
    """The oracle's environment emitter (environment.cpp) loaded from an OpenEXR file."""

    def __init__(self, path, strength=1.0):
        self.h = lib().orc_env_load(os.fsencode(path), strength)
        if not self.h:
            raise RuntimeError("cannot load environment map %s" % path)

    def sample(self, u):
        u = np.ascontiguousarray(u, dtype=np.float32).reshape(-1, 2)
        n = u.shape[0]
        d, p, L = np.zeros((n, 3), np.float32), np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
        lib().orc_env_sample(self.h, n, _fp(u), _fp(d), _fp(p), _fp(L))
        return d, p, L

    def pdf(self, dirs):
        d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
        p = np.zeros(d.shape[0], np.float32)
        lib().orc_env_pdf(self.h, d.shape[0], _fp(d), _fp(p))
        return p

    def eval(self, dirs):
        d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
        L = np.zeros((d.shape[0], 3), np.float32)
        lib().orc_env_eval(self.h, d.shape[0], _fp(d), _fp(L))
        return L

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_env_free(self.h)
            self.h = None


def motion_interpolate(a, b, t):
    """AnimatedTransform::interpolate between 4x4 matrices a (time 0) and b (time 1):
    returns the 3x4 matrix at time t and its inverse."""
    a = np.ascontiguousarray(a, np.float32).reshape(4, 4)
    b = np.ascontiguousarray(b, np.float32).reshape(4, 4)
    m = np.zeros((3, 4), np.float32)
    mi = np.zeros((3, 4), np.float32)
    lib().orc_motion_interpolate(_fp(a), _fp(b), t, _fp(m), _fp(mi))
    return m, mi


def tex_eval(xml_path, p, n=None, dpdu=None, uv=None):
    """Evaluates the texture that is the root element of `xml_path` at surface points
    (p, n, dpdu, uv); returns rgb per point (float textures repeat their value)."""
    p = np.asarray(p, np.float32).reshape(-1, 3)
    k = p.shape[0]
    pts = np.zeros((k, 11), np.float32)
    pts[:, 0:3] = p
    pts[:, 3:6] = (0, 0, 1) if n is None else np.asarray(n, np.float32).reshape(-1, 3)
    pts[:, 6:9] = (1, 0, 0) if dpdu is None else np.asarray(dpdu, np.float32).reshape(-1, 3)
    pts[:, 9:11] = 0 if uv is None else np.asarray(uv, np.float32).reshape(-1, 2)
    out = np.zeros((k, 3), np.float32)
    err = ctypes.create_string_buffer(512)
    if lib().orc_tex_eval(os.fsencode(xml_path), k, _fp(pts), _fp(out), err, 512) != 0:
        raise RuntimeError(err.value.decode())
    return out


def perlin_perm():
    out = np.zeros(512, np.int32)
    lib().orc_perlin_perm(out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    return out
