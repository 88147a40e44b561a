"""gianduia_b200: B200-native radiance path (BVH4 traversal + path/volpath wavefront
integrators) for Gianduia scenes.

Python binding of the C ABI in include/gnd_gpu.h (libgianduia_b200.so, built in-tree by
gianduia_b200/build.py). The compute path is the CUDA library only: when no CUDA device
is usable the GPU calls fail with GpuUnavailable; nothing falls back to the CPU.
"""
import ctypes
import os
import threading

import numpy as np

from . import build as _build

__all__ = ["lib", "HostScene", "GpuContext", "GndError", "GpuUnavailable", "RAY_DTYPE", "HIT_DTYPE"]

GND_OK = 0
GND_ERR_INVALID = 1
GND_ERR_TIMEOUT = 5
GND_ERR_CANCELLED = 7
GND_ERR_BUDGET = 8
GND_ERR_NO_DEVICE = 9
GND_HOST_DEVICE_BLAS = 1
_STATUS = {1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "device check failed",
           5: "timeout", 6: "parse error", 7: "cancelled", 8: "over HBM budget", 9: "no CUDA device"}

RAY_DTYPE = np.dtype([("o", np.float32, 3), ("tmin", np.float32), ("d", np.float32, 3), ("tmax", np.float32)])
HIT_DTYPE = np.dtype([("t", np.float32), ("u", np.float32), ("v", np.float32), ("inst", np.int32), ("prim", np.int32)])
# Camera record of a flattened scene (gnd::Camera, 112 bytes): kind 0 pinhole, 1 thin lens
CAMERA_DTYPE = np.dtype([("to_world", np.float32, (3, 4)), ("width", np.int32), ("height", np.int32),
                         ("scale", np.float32), ("aspect", np.float32), ("origin", np.float32, 3), ("pad", np.float32),
                         ("kind", np.int32), ("blades", np.int32), ("lens_radius", np.float32),
                         ("focal_distance", np.float32), ("k1", np.float32), ("ca_axial", np.float32),
                         ("ca_lateral", np.float32), ("vignetting", np.int32), ("rolling_shutter", np.int32),
                         ("scan_duration", np.float32), ("exposure_duration", np.float32), ("animated", np.int32),
                         ("motion", np.float32, 48)])
assert CAMERA_DTYPE.itemsize == 320
# BVH4 node (gnd::Node4): child bounds as rows lox, hix, loy, hiy, loz, hiz
NODE_DTYPE = np.dtype([("lo_hi", np.float32, (6, 4)), ("child", np.uint32, 4), ("pad", np.uint32, 4)])


class GndError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d: %s)" % (msg, status, _STATUS.get(status, "?")))
        self.status = status


class GpuUnavailable(GndError):
    pass


_lib = None
_lock = threading.Lock()
_vp = ctypes.c_void_p


def lib():
    """Loads libgianduia_b200.so (building it first when the sources changed)."""
    global _lib
    with _lock:
        if _lib is None:
            path = _build.build()
            L = ctypes.CDLL(path)
            L.gnd_last_error.restype = ctypes.c_char_p
            L.gnd_version.restype = ctypes.c_char_p
            for name, args in {
                "gnd_host_load_xml": [ctypes.c_char_p, ctypes.POINTER(_vp)],
                "gnd_host_from_triangles": [_vp, ctypes.c_int64, ctypes.POINTER(_vp)],
                "gnd_host_load_xml_ex": [ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(_vp)],
                "gnd_host_from_triangles_ex": [_vp, ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(_vp)],
                "gnd_gpu_scene_info": [_vp, ctypes.c_uint64, _vp],
                "gnd_gpu_set_build_leaf_max": [_vp, ctypes.c_int32],
                "gnd_gpu_post": [_vp, _vp, ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp],
                "gnd_gpu_post_dev": [_vp, _vp, ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp, _vp],
                "gnd_image_write_png": [ctypes.c_char_p, _vp, ctypes.c_int32, ctypes.c_int32],
                "gnd_image_write_exr": [ctypes.c_char_p, _vp, ctypes.c_int32, ctypes.c_int32],
                "gnd_image_read_exr": [ctypes.c_char_p, _vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int32),
                                       ctypes.POINTER(ctypes.c_int32)],
                "gnd_gpu_scene_download": [_vp, ctypes.c_uint64, ctypes.c_int32, _vp, ctypes.c_int64],
                "gnd_gpu_scene_refit_mesh": [_vp, ctypes.c_uint64, ctypes.c_int32, _vp, ctypes.c_int64, _vp],
                "gnd_host_scene_desc": [_vp, ctypes.POINTER(_vp)],
                "gnd_host_free": [_vp],
                "gnd_gpu_create": [ctypes.c_int, ctypes.POINTER(_vp)],
                "gnd_gpu_destroy": [_vp],
                "gnd_gpu_scene_upload": [_vp, _vp, ctypes.POINTER(ctypes.c_uint64)],
                "gnd_gpu_scene_free": [_vp, ctypes.c_uint64],
                "gnd_gpu_host_register": [_vp, ctypes.c_int32],
                "gnd_gpu_scene_bytes": [_vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)],
                "gnd_gpu_trace_closest": [_vp, ctypes.c_uint64, _vp, ctypes.c_int64, _vp],
                "gnd_gpu_trace_any": [_vp, ctypes.c_uint64, _vp, ctypes.c_int64, _vp],
                "gnd_gpu_trace_closest_dev": [_vp, ctypes.c_uint64, _vp, ctypes.c_int64, _vp, _vp],
                "gnd_gpu_trace_any_dev": [_vp, ctypes.c_uint64, _vp, ctypes.c_int64, _vp, _vp],
                "gnd_gpu_trace_count_dev": [_vp, ctypes.c_uint64, _vp, ctypes.c_int64, _vp, _vp, _vp],
                "gnd_gpu_render": [_vp, ctypes.c_uint64, _vp, _vp, _vp],
                "gnd_gpu_render_fixed": [_vp, ctypes.c_uint64, _vp, _vp, _vp, _vp],
                "gnd_gpu_counters": [_vp, _vp, ctypes.c_int32],
                "gnd_gpu_cancel": [_vp],
                "gnd_gpu_trace_closest_fixed": [_vp, ctypes.c_uint64, _vp, ctypes.c_int64, _vp],
                "gnd_gpu_set_hbm_budget": [_vp, ctypes.c_uint64],
                "gnd_gpu_serve_submit": [_vp, _vp, ctypes.POINTER(ctypes.c_uint64)],
                "gnd_gpu_serve_poll": [_vp, ctypes.c_uint64, _vp],
                "gnd_gpu_serve_wait": [_vp, ctypes.c_uint64, _vp, _vp, ctypes.c_int64],
                "gnd_gpu_serve_cancel": [_vp, ctypes.c_uint64],
                "gnd_gpu_serve_policy": [_vp, ctypes.c_int32],
                "gnd_gpu_serve_tune": [_vp, _vp],
                "gnd_gpu_read_bandwidth": [_vp, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)],
                "gnd_gpu_get_tune": [_vp, ctypes.c_uint64, _vp],
                "gnd_gpu_set_tune": [_vp, ctypes.c_uint64, _vp],
                "gnd_gpu_autotune": [_vp, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32, _vp, ctypes.POINTER(ctypes.c_double)],
            }.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = ctypes.c_int32
            _lib = L
    return _lib


def _check(status, what):
    if status != GND_OK:
        msg = "%s: %s" % (what, lib().gnd_last_error().decode(errors="replace"))
        if status == GND_ERR_NO_DEVICE:
            raise GpuUnavailable(status, msg)
        raise GndError(status, msg)


class PostParams(ctypes.Structure):
    _fields_ = [("tonemapper", ctypes.c_int32), ("exposure", ctypes.c_float), ("bloom", ctypes.c_int32),
                ("bloom_threshold", ctypes.c_float), ("bloom_radius", ctypes.c_float),
                ("bloom_intensity", ctypes.c_float), ("bloom_mips", ctypes.c_int32), ("output", ctypes.c_int32)]


TONEMAPPERS = {"linear": 0, "reinhard": 1, "uncharted2": 2, "aces": 3, "khronos_pbr": 4, "agx": 5, "agx_punchy": 6}


def post_params(tonemapper=0, exposure=0.0, bloom=False, threshold=1.0, radius=1.0, intensity=0.04, mips=6, output=0):
    """gnd_post_params with the reference PostProcessor's defaults."""
    if isinstance(tonemapper, str):
        tonemapper = TONEMAPPERS[tonemapper]
    return PostParams(tonemapper, exposure, 1 if bloom else 0, threshold, radius, intensity, mips, output)


def write_png(path, rgb8):
    """Film::savePNG's file: an 8-bit RGB image [h, w, 3]."""
    a = np.ascontiguousarray(rgb8, dtype=np.uint8)
    _check(lib().gnd_image_write_png(os.fsencode(path), a.ctypes.data, a.shape[1], a.shape[0]), "gnd_image_write_png")


def write_exr(path, rgb):
    """Film::saveEXR's file: a float RGB image [h, w, 3]."""
    a = np.ascontiguousarray(rgb, dtype=np.float32)
    _check(lib().gnd_image_write_exr(os.fsencode(path), a.ctypes.data, a.shape[1], a.shape[0]), "gnd_image_write_exr")


def read_exr(path):
    """A scanline OpenEXR image (compression none, ZIPS or ZIP) as float RGB [h, w, 3]."""
    w, h = ctypes.c_int32(), ctypes.c_int32()
    _check(lib().gnd_image_read_exr(os.fsencode(path), None, 0, ctypes.byref(w), ctypes.byref(h)), "gnd_image_read_exr")
    out = np.zeros((h.value, w.value, 3), np.float32)
    _check(lib().gnd_image_read_exr(os.fsencode(path), out.ctypes.data, out.nbytes, ctypes.byref(w), ctypes.byref(h)),
           "gnd_image_read_exr")
    return out


class SceneInfo(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int64), ("num_tris", ctypes.c_int64), ("num_instances", ctypes.c_int32),
                ("blas_on_device", ctypes.c_int32), ("fast_boxes", ctypes.c_int32), ("num_meshes", ctypes.c_int32),
                ("build_ms", ctypes.c_double), ("bytes", ctypes.c_uint64)]


class SceneDesc(ctypes.Structure):
    """Mirror of gnd_scene_desc (read-only view of the render settings)."""
    _fields_ = [
        ("nodes", _vp), ("num_nodes", ctypes.c_int64), ("tris", _vp), ("tri_attrs", _vp), ("num_tris", ctypes.c_int64),
        ("inst_trav", _vp), ("inst_shade", _vp), ("num_instances", ctypes.c_int32), ("tlas_root", ctypes.c_uint32),
        ("tlas_list", _vp), ("tlas_list_len", ctypes.c_int64), ("materials", _vp), ("num_materials", ctypes.c_int32),
        ("num_emitters", ctypes.c_int32), ("emitters", _vp), ("media", _vp), ("num_media", ctypes.c_int32),
        ("num_meshes", ctypes.c_int32), ("meshes", _vp), ("cdf", _vp), ("cdf_len", ctypes.c_int64),
        ("orig_to_leaf", _vp), ("orig_to_leaf_len", ctypes.c_int64), ("camera", _vp),
        ("width", ctypes.c_int32), ("height", ctypes.c_int32), ("spp", ctypes.c_int32), ("max_depth", ctypes.c_int32),
        ("integrator", ctypes.c_int32), ("filter", ctypes.c_int32), ("filter_radius", ctypes.c_float * 2),
        ("filter_alpha", ctypes.c_float), ("blas_on_device", ctypes.c_int32),
        ("env_emitter", ctypes.c_int32), ("env_width", ctypes.c_int32), ("env_height", ctypes.c_int32),
        ("env_marginal_integral", ctypes.c_float), ("env_strength", ctypes.c_float), ("pad2", ctypes.c_int32),
        ("env_texels", _vp), ("env_dist", _vp), ("inst_motion", _vp),
        ("tex_nodes", _vp), ("num_tex_nodes", ctypes.c_int32), ("pad3", ctypes.c_int32),
        ("tex_texels", _vp), ("num_tex_texels", ctypes.c_int64),
    ]


class HostScene:
    """A scene parsed, BVH-built and flattened by the host framework (no GPU needed)."""

    def __init__(self, handle):
        self._h = _vp(handle)
        d = _vp()
        _check(lib().gnd_host_scene_desc(self._h, ctypes.byref(d)), "gnd_host_scene_desc")
        self._desc_ptr = d
        self.desc = SceneDesc.from_address(d.value)

    @staticmethod
    def load_xml(path, device_blas=False):
        """Parses and flattens a scene file. device_blas: leave the mesh trees to the GPU
        (built at upload) instead of the host SAH builder."""
        h = _vp()
        flags = GND_HOST_DEVICE_BLAS if device_blas else 0
        _check(lib().gnd_host_load_xml_ex(os.fsencode(path), flags, ctypes.byref(h)), "gnd_host_load_xml(%s)" % path)
        return HostScene(h.value)

    @staticmethod
    def from_triangles(tris, device_blas=False):
        tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
        h = _vp()
        flags = GND_HOST_DEVICE_BLAS if device_blas else 0
        _check(lib().gnd_host_from_triangles_ex(tris.ctypes.data, tris.shape[0], flags, ctypes.byref(h)),
               "gnd_host_from_triangles")
        return HostScene(h.value)

    def camera(self):
        """The flattened camera record (CAMERA_DTYPE), or None for a scene without one."""
        if not self.desc.camera:
            return None
        return np.frombuffer(ctypes.string_at(self.desc.camera, CAMERA_DTYPE.itemsize), CAMERA_DTYPE)[0]

    def pin(self, on=True):
        """Page-locks (or releases) the large host arrays so uploads run at DMA speed."""
        _check(lib().gnd_gpu_host_register(self._desc_ptr, 1 if on else 0), "gnd_gpu_host_register")
        self._pinned = bool(on)

    def close(self):
        if self._h and self._h.value:
            if getattr(self, "_pinned", False):
                lib().gnd_gpu_host_register(self._desc_ptr, 0)
                self._pinned = False
            lib().gnd_host_free(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def width(self):
        return self.desc.width

    @property
    def height(self):
        return self.desc.height

    @property
    def spp(self):
        return self.desc.spp

    def nodes(self):
        """The flattened BVH4 nodes as a structured numpy view (copy)."""
        dt = NODE_DTYPE
        n = self.desc.num_nodes
        buf = (ctypes.c_char * (n * 128)).from_address(self.desc.nodes)
        return np.frombuffer(bytes(buf), dtype=dt)

    def tris(self):
        n = self.desc.num_tris
        buf = (ctypes.c_char * (n * 48)).from_address(self.desc.tris)
        return np.frombuffer(bytes(buf), dtype=np.float32).reshape(n, 12)

    def tlas_list(self):
        n = self.desc.tlas_list_len
        return np.ctypeslib.as_array((ctypes.c_uint32 * n).from_address(self.desc.tlas_list)).copy() if n else np.zeros(0, np.uint32)

    def inst_trav(self):
        n = self.desc.num_instances
        buf = (ctypes.c_char * (n * 64)).from_address(self.desc.inst_trav)
        return np.frombuffer(bytes(buf), dtype=np.uint32).reshape(n, 16)


def as_rays(arr):
    """(n, 8) float32 (ox, oy, oz, tmin, dx, dy, dz, tmax) -> contiguous gnd_ray array."""
    a = np.ascontiguousarray(arr, dtype=np.float32).reshape(-1, 8)
    return a


class GpuContext:
    """One CUDA device (gnd_gpu_create). Raises GpuUnavailable without a usable B200."""

    def __init__(self, device=0):
        self._h = _vp()
        _check(lib().gnd_gpu_create(device, ctypes.byref(self._h)), "gnd_gpu_create")
        self._scenes = {}

    def close(self):
        if self._h and self._h.value:
            lib().gnd_gpu_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def upload(self, host_scene):
        sid = ctypes.c_uint64()
        _check(lib().gnd_gpu_scene_upload(self._h, host_scene._desc_ptr, ctypes.byref(sid)), "gnd_gpu_scene_upload")
        self._scenes[sid.value] = host_scene
        return sid.value

    def free_scene(self, sid):
        _check(lib().gnd_gpu_scene_free(self._h, sid), "gnd_gpu_scene_free")
        self._scenes.pop(sid, None)

    def scene_bytes(self, sid):
        b = ctypes.c_uint64()
        _check(lib().gnd_gpu_scene_bytes(self._h, sid, ctypes.byref(b)), "gnd_gpu_scene_bytes")
        return b.value

    def set_build_leaf_max(self, leaf_max):
        """Largest leaf of mesh trees built on the GPU by later uploads (1..16)."""
        _check(lib().gnd_gpu_set_build_leaf_max(self._h, leaf_max), "gnd_gpu_set_build_leaf_max")

    def post(self, rgb, want_hdr=True, want_rgb8=True, **params):
        """Post-processing of a linear image [h, w, 3] on the GPU (gnd_gpu_post): returns
        (tonemapped float image or None, 8-bit image or None). Keyword arguments as
        post_params."""
        a = np.ascontiguousarray(rgb, dtype=np.float32)
        h, w = a.shape[:2]
        hdr = np.zeros((h, w, 3), np.float32) if want_hdr else None
        out8 = np.zeros((h, w, 3), np.uint8) if want_rgb8 else None
        p = post_params(**params)
        _check(lib().gnd_gpu_post(self._h, a.ctypes.data, w, h, ctypes.byref(p),
                                  hdr.ctypes.data if hdr is not None else None,
                                  out8.ctypes.data if out8 is not None else None), "gnd_gpu_post")
        return hdr, out8

    def scene_info(self, sid):
        """Sizes and build record of an uploaded scene (gnd_gpu_scene_info) as a dict."""
        info = SceneInfo()
        _check(lib().gnd_gpu_scene_info(self._h, sid, ctypes.byref(info)), "gnd_gpu_scene_info")
        return {k: getattr(info, k) for k, _ in SceneInfo._fields_}

    def refit_mesh(self, sid, mesh, positions):
        """New object-space positions (triangles x 9 floats, the mesh's original triangle
        order) for mesh `mesh`; its tree and the top-level tree are refitted on the GPU
        (gnd_gpu_scene_refit_mesh). Returns the device time in ms."""
        pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 9)
        ms = ctypes.c_float()
        _check(lib().gnd_gpu_scene_refit_mesh(self._h, sid, mesh, pos.ctypes.data, pos.shape[0], ctypes.byref(ms)),
               "gnd_gpu_scene_refit_mesh")
        return ms.value

    def download(self, sid, array):
        """One device array of an uploaded scene (gnd_gpu_scene_download): "nodes",
        "tris", "tri_attrs", "orig_to_leaf" or "inst_trav", as raw numpy records."""
        info = self.scene_info(sid)
        code, dt, n = {
            "nodes": (0, NODE_DTYPE, info["num_nodes"]),
            "tris": (1, np.dtype((np.float32, 12)), info["num_tris"]),
            "tri_attrs": (2, np.dtype((np.float32, 16)), info["num_tris"]),
            "orig_to_leaf": (3, np.dtype(np.uint32), info["num_tris"]),
            "inst_trav": (4, np.dtype((np.float32, 16)), info["num_instances"]),
        }[array]
        out = np.zeros(n, dt)
        _check(lib().gnd_gpu_scene_download(self._h, sid, code, out.ctypes.data, out.nbytes), "gnd_gpu_scene_download")
        return out

    def trace_closest(self, sid, rays):
        r = as_rays(rays)
        hits = np.zeros(r.shape[0], HIT_DTYPE)
        _check(lib().gnd_gpu_trace_closest(self._h, sid, r.ctypes.data, r.shape[0], hits.ctypes.data), "gnd_gpu_trace_closest")
        return hits

    def trace_any(self, sid, rays):
        r = as_rays(rays)
        occ = np.zeros(r.shape[0], np.uint8)
        _check(lib().gnd_gpu_trace_any(self._h, sid, r.ctypes.data, r.shape[0], occ.ctypes.data), "gnd_gpu_trace_any")
        return occ.astype(bool)

    # device-pointer variants (pointers as ints, e.g. torch tensor.data_ptr())
    def trace_closest_dev(self, sid, d_rays, n, d_hits, stream=0):
        _check(lib().gnd_gpu_trace_closest_dev(self._h, sid, d_rays, n, d_hits, stream or None), "gnd_gpu_trace_closest_dev")

    def trace_any_dev(self, sid, d_rays, n, d_occ, stream=0):
        _check(lib().gnd_gpu_trace_any_dev(self._h, sid, d_rays, n, d_occ, stream or None), "gnd_gpu_trace_any_dev")

    def trace_count_dev(self, sid, d_rays, n, d_nodes, d_tris, stream=0):
        _check(lib().gnd_gpu_trace_count_dev(self._h, sid, d_rays, n, d_nodes, d_tris, stream or None), "gnd_gpu_trace_count_dev")

    def _film_size(self, sid, width, height):
        hs = self._scenes[sid]
        return (width if width > 0 else hs.width), (height if height > 0 else hs.height)

    def render(self, sid, spp=0, first_pass=0, max_depth=0, integrator=-1, window=None, batched=False, film=None,
               callback=None, profile=0, width=0, height=0):
        """gnd_gpu_render: adds passes [first_pass, first_pass + spp) of the scene into
        `film` (float32 [H, W, 7]: sum wL rgb, sum w, sum wL^2 rgb). Returns (film, stats).
        width / height override the scene file's film size."""
        W, H = self._film_size(sid, width, height)
        if film is None:
            film = np.zeros((H, W, 7), np.float32)
        assert film.dtype == np.float32 and film.shape == (H, W, 7) and film.flags.c_contiguous
        p = self._params(spp, first_pass, max_depth, integrator, window, batched, profile, width, height)
        cb = None
        if callback is not None:
            def _cb(user, s, fptr, w, h):
                arr = np.ctypeslib.as_array(fptr, shape=(h, w, 7)).copy()
                callback(int(s), arr)
            cb = PROGRESS_FN(_cb)
            p.callback = cb
        st = RenderStats()
        _check(lib().gnd_gpu_render(self._h, sid, ctypes.byref(p), film.ctypes.data, ctypes.byref(st)), "gnd_gpu_render")
        return film, st.as_dict()

    def render_fixed(self, sid, spp=0, first_pass=0, max_depth=0, integrator=-1, window=None, batched=False, fsum=None,
                     fsq=None, profile=0, width=0, height=0):
        """gnd_gpu_render_fixed: adds the passes into the exact film -- fsum (uint64 [H, W, 4],
        sum wL rgb and sum w in units of 2^-24) and fsq (float32 [H, W, 3], sum wL^2).
        Returns (fsum, fsq, stats)."""
        W, H = self._film_size(sid, width, height)
        if fsum is None:
            fsum = np.zeros((H, W, 4), np.uint64)
        if fsq is None:
            fsq = np.zeros((H, W, 3), np.float32)
        assert fsum.dtype == np.uint64 and fsum.shape == (H, W, 4) and fsum.flags.c_contiguous
        assert fsq.dtype == np.float32 and fsq.shape == (H, W, 3) and fsq.flags.c_contiguous
        p = self._params(spp, first_pass, max_depth, integrator, window, batched, profile, width, height)
        st = RenderStats()
        _check(lib().gnd_gpu_render_fixed(self._h, sid, ctypes.byref(p), fsum.ctypes.data, fsq.ctypes.data,
                                          ctypes.byref(st)), "gnd_gpu_render_fixed")
        return fsum, fsq, st.as_dict()

    def counters(self, reset=False):
        """gnd_gpu_counters: the context's work counters as a dict (`last`: the last render's stats)."""
        c = Counters()
        _check(lib().gnd_gpu_counters(self._h, ctypes.byref(c), 1 if reset else 0), "gnd_gpu_counters")
        d = {name: getattr(c, name) for name, _ in Counters._fields_ if name != "last"}
        d["last"] = c.last.as_dict()
        return d

    @staticmethod
    def _params(spp, first_pass, max_depth, integrator, window, batched, profile, width, height):
        p = RenderParams()
        p.spp = spp
        p.first_pass = first_pass
        p.max_depth = max_depth
        p.integrator = integrator
        if window is not None:
            p.window[:] = list(window)
        p.batched = 1 if batched else 0
        p.profile = profile
        p.width = width
        p.height = height
        return p

    def cancel(self):
        _check(lib().gnd_gpu_cancel(self._h), "gnd_gpu_cancel")

    # ---- serving (gnd_gpu_serve_*)
    # ---- engine settings (gnd_tune)
    def get_tune(self, sid):
        t = Tune()
        _check(lib().gnd_gpu_get_tune(self._h, sid, ctypes.byref(t)), "gnd_gpu_get_tune")
        return t.as_dict()

    def set_tune(self, sid, **fields):
        t = Tune()
        _check(lib().gnd_gpu_get_tune(self._h, sid, ctypes.byref(t)), "gnd_gpu_get_tune")
        for k, v in fields.items():
            setattr(t, k, int(v))
        _check(lib().gnd_gpu_set_tune(self._h, sid, ctypes.byref(t)), "gnd_gpu_set_tune")

    def autotune(self, sid, spp=8, budget_ms=4000):
        """Measures engine settings for the scene (gnd_gpu_autotune); returns (settings, Mpaths/s)."""
        t = Tune()
        m = ctypes.c_double()
        _check(lib().gnd_gpu_autotune(self._h, sid, int(spp), int(budget_ms), ctypes.byref(t), ctypes.byref(m)),
               "gnd_gpu_autotune")
        return t.as_dict(), m.value

    def read_bandwidth(self, nbytes, reps):
        """GB/s of L2-cached 16-byte loads streaming a buffer of nbytes, reps times."""
        g = ctypes.c_double()
        _check(lib().gnd_gpu_read_bandwidth(self._h, int(nbytes), int(reps), ctypes.byref(g)), "gnd_gpu_read_bandwidth")
        return g.value

    def serve_policy(self, policy):
        """'deadline' (earliest submission + 4x estimated render time first, the default),
        'srpt' (fewest samples left to hand out first) or 'fifo' (oldest job first)."""
        code = {"fifo": 0, "srpt": 1, "deadline": 2}[policy]
        _check(lib().gnd_gpu_serve_policy(self._h, code), "gnd_gpu_serve_policy")

    def serve_tune(self, **fields):
        """Engine settings of the serving thread (the defaults of gnd_tune, updated by fields)."""
        t = Tune(pool_log2=22, round_iters=4, trav_blocks=8, material_sort=1, stack_smem=32, graphs=1, sample_film=1,
                 spec_extend=0, spec_shadow=0, ray_sort=0, leaf_batch=32, trace_leaf_batch=12,
                 shadow_leaf_batch=32, trace_blocks=8)
        for k, v in fields.items():
            setattr(t, k, int(v))
        _check(lib().gnd_gpu_serve_tune(self._h, ctypes.byref(t)), "gnd_gpu_serve_tune")

    def set_hbm_budget(self, nbytes):
        _check(lib().gnd_gpu_set_hbm_budget(self._h, int(nbytes)), "gnd_gpu_set_hbm_budget")

    def submit(self, sid, width=0, height=0, spp=0, max_depth=0, integrator=-1, first_pass=0):
        """Queues a render job; returns its id at once."""
        d = JobDesc(scene=sid, width=width, height=height, spp=spp, max_depth=max_depth, integrator=integrator,
                    first_pass=first_pass)
        jid = ctypes.c_uint64()
        _check(lib().gnd_gpu_serve_submit(self._h, ctypes.byref(d), ctypes.byref(jid)), "gnd_gpu_serve_submit")
        w = width if width > 0 else self._scenes[sid].width
        h = height if height > 0 else self._scenes[sid].height
        self._jobs = getattr(self, "_jobs", {})
        self._jobs[jid.value] = (h, w)
        return jid.value

    def poll(self, jid):
        st = JobStatus()
        _check(lib().gnd_gpu_serve_poll(self._h, jid, ctypes.byref(st)), "gnd_gpu_serve_poll")
        return st.as_dict()

    def wait(self, jid, timeout_ms=-1):
        """Blocks until the job finishes; returns (film [H, W, 7], status dict). A cancelled
        or failed job raises GndError; wait_any returns its status code instead."""
        h, w = self._jobs[jid]
        film = np.zeros((h, w, 7), np.float32)
        st = JobStatus()
        _check(lib().gnd_gpu_serve_wait(self._h, jid, film.ctypes.data, ctypes.byref(st), int(timeout_ms)),
               "gnd_gpu_serve_wait")
        del self._jobs[jid]
        return film, st.as_dict()

    def wait_any(self, jid, timeout_ms=-1):
        """As wait, but returns (film, status, gnd_status) instead of raising."""
        h, w = self._jobs[jid]
        film = np.zeros((h, w, 7), np.float32)
        st = JobStatus()
        rc = lib().gnd_gpu_serve_wait(self._h, jid, film.ctypes.data, ctypes.byref(st), int(timeout_ms))
        if rc != GND_ERR_TIMEOUT:
            del self._jobs[jid]
        return film, st.as_dict(), rc

    def cancel_job(self, jid):
        _check(lib().gnd_gpu_serve_cancel(self._h, jid), "gnd_gpu_serve_cancel")


PROGRESS_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_float), ctypes.c_int32,
                               ctypes.c_int32)


class RenderParams(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_int32), ("first_pass", ctypes.c_int32), ("max_depth", ctypes.c_int32),
                ("integrator", ctypes.c_int32), ("window", ctypes.c_int32 * 4), ("batched", ctypes.c_int32),
                ("profile", ctypes.c_int32), ("callback", PROGRESS_FN), ("user", _vp), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32)]


class RenderStats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_int64), ("rays", ctypes.c_int64), ("passes_done", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("ms", ctypes.c_double), ("extend_rays", ctypes.c_int64),
                ("shadow_rays", ctypes.c_int64), ("extend_nodes", ctypes.c_int64), ("extend_tris", ctypes.c_int64),
                ("extend_ms", ctypes.c_double), ("iterations", ctypes.c_int64), ("launches", ctypes.c_int64),
                ("extend_node_warp_steps", ctypes.c_int64), ("extend_leaf_steps", ctypes.c_int64),
                ("extend_leaf_warp_steps", ctypes.c_int64)]

    def as_dict(self):
        return dict(paths=self.paths, rays=self.rays, passes=self.passes_done, ms=self.ms, extend_rays=self.extend_rays,
                    shadow_rays=self.shadow_rays, extend_nodes=self.extend_nodes, extend_tris=self.extend_tris,
                    extend_ms=self.extend_ms, iterations=self.iterations, launches=self.launches,
                    extend_node_warp_steps=self.extend_node_warp_steps, extend_leaf_steps=self.extend_leaf_steps,
                    extend_leaf_warp_steps=self.extend_leaf_warp_steps)


class Counters(ctypes.Structure):
    """gnd_counters"""
    _fields_ = [("trace_batches", ctypes.c_int64), ("trace_rays", ctypes.c_int64), ("counted_rays", ctypes.c_int64),
                ("counted_nodes", ctypes.c_int64), ("counted_tris", ctypes.c_int64), ("renders", ctypes.c_int64),
                ("paths", ctypes.c_int64), ("extend_rays", ctypes.c_int64), ("shadow_rays", ctypes.c_int64),
                ("extend_nodes", ctypes.c_int64), ("extend_tris", ctypes.c_int64), ("iterations", ctypes.c_int64),
                ("launches", ctypes.c_int64), ("render_ms", ctypes.c_double), ("last", RenderStats)]


class Tune(ctypes.Structure):
    _fields_ = [("pool_log2", ctypes.c_int32), ("round_iters", ctypes.c_int32), ("trav_blocks", ctypes.c_int32),
                ("material_sort", ctypes.c_int32), ("stack_smem", ctypes.c_int32), ("graphs", ctypes.c_int32),
                ("sample_film", ctypes.c_int32), ("spec_extend", ctypes.c_int32), ("spec_shadow", ctypes.c_int32),
                ("ray_sort", ctypes.c_int32), ("leaf_batch", ctypes.c_int32), ("trace_leaf_batch", ctypes.c_int32),
                ("shadow_leaf_batch", ctypes.c_int32), ("trace_blocks", ctypes.c_int32)]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class JobDesc(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_uint64), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("spp", ctypes.c_int32), ("max_depth", ctypes.c_int32), ("integrator", ctypes.c_int32),
                ("first_pass", ctypes.c_int32)]


JOB_STATES = {0: "queued", 1: "running", 2: "done", 3: "cancelled", 4: "failed"}


class JobStatus(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("pad", ctypes.c_int32), ("samples_total", ctypes.c_int64),
                ("samples_done", ctypes.c_int64), ("submit_ms", ctypes.c_double), ("admit_ms", ctypes.c_double),
                ("done_ms", ctypes.c_double)]

    def as_dict(self):
        return dict(state=JOB_STATES.get(self.state, self.state), samples_total=self.samples_total,
                    samples_done=self.samples_done, submit_ms=self.submit_ms, admit_ms=self.admit_ms,
                    done_ms=self.done_ms)


def resolve(film):
    """Image = sum(w L) / sum(w) per pixel (film.cpp:50-95)."""
    w = film[..., 3:4]
    return np.where(w > 0, film[..., :3] / np.maximum(w, 1e-30), 0.0).astype(np.float32)


def fixed_to_film(fsum, fsq):
    """The float film [H, W, 7] of an exact film (fsum uint64 [H, W, 4] in units of 2^-24,
    fsq float32 [H, W, 3]), converted as gnd_gpu_render converts it."""
    f = np.empty(fsum.shape[:2] + (7,), np.float32)
    f[..., :4] = (fsum.astype(np.float64) * (1.0 / 16777216.0)).astype(np.float32)
    f[..., 4:] = fsq
    return f
