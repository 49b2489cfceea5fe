"""ctypes binding of the CPU oracle (liboracle.so), its double-precision build (liboracle_fp64.so, the
ground truth of error measurements) and of the reference harness (librefcpu.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from piper2_b200 import capi  # noqa: E402  (struct layouts of include/piper2_b200.h)

ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
ORACLE64_SO = os.path.join(HERE, "_build", "liboracle_fp64.so")
REF_SO = os.path.join(HERE, "_ref", "librefcpu.so")

_or = None
_or64 = None
_ref = None


def _load(path):
    # (re)build when missing or older than its sources (a no-op otherwise): the library reads the C ABI's structs,
    # so a stale build would misread them
    sys.path.insert(0, HERE)
    from build_oracle import build_oracle as _b

    _b()
    return C.CDLL(path)


def oracle():
    global _or
    if _or is None:
        h = _load(ORACLE_SO)
        h.or_sobol_sample.restype = C.c_float
        h.or_sobol_sample.argtypes = [C.c_uint64, C.c_uint32]
        h.or_conv.restype = None
        h.or_conv.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32]
        h.or_sobol_sample_scrambled.restype = C.c_float
        h.or_sobol_sample_scrambled.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        h.or_sobol_interval_to_index.restype = C.c_uint64
        h.or_sobol_interval_to_index.argtypes = [C.c_uint32] * 4
        h.or_sobol_start.argtypes = [C.c_uint32] * 5 + [C.POINTER(C.c_uint64), C.POINTER(C.c_float)]
        h.or_sobol_digest.restype = C.c_char_p
        h.or_remap_roughness.restype = C.c_float
        h.or_remap_roughness.argtypes = [C.c_float]
        h.or_logf.restype = C.c_float
        h.or_logf.argtypes = [C.c_float]
        h.or_remap_roughness_point.restype = C.c_float
        h.or_remap_roughness_point.argtypes = [C.c_float]
        h.or_texture_sample.argtypes = [C.POINTER(capi.Texture), C.c_float, C.c_float, C.POINTER(C.c_float)]
        h.or_camera_ray.argtypes = [C.POINTER(capi.Camera), C.c_float, C.c_float, C.c_float, C.c_float,
                                    C.POINTER(capi.Ray)]
        h.or_scene_create.restype = C.c_void_p
        h.or_scene_create.argtypes = [C.POINTER(capi.Scene), C.c_int]
        h.or_scene_destroy.argtypes = [C.c_void_p]
        h.or_scene_triangle_count.restype = C.c_uint32
        h.or_scene_triangle_count.argtypes = [C.c_void_p]
        h.or_trace_closest.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int]
        h.or_trace_any.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int]
        h.or_trace_counters.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.POINTER(C.c_uint64),
                                        C.POINTER(C.c_uint64)]
        h.or_render.restype = C.c_int
        h.or_render.argtypes = [C.c_void_p, C.POINTER(capi.RenderSettings), C.POINTER(capi.Rect), C.c_uint32,
                                C.c_uint32, C.c_void_p, C.c_void_p, C.c_int]
        h.or_bsdf_sample.argtypes = [C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
        h.or_bsdf_eval.argtypes = [C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
        h.or_calc_render_rect.argtypes = [C.c_uint32, C.c_uint32, C.c_float, C.c_uint32,
                                          C.POINTER(capi.NDCTransform), C.POINTER(capi.Rect)]
        h.or_plane_make.argtypes = [C.POINTER(C.c_float)] * 3 + [C.POINTER(capi.Plane)]
        h.or_intersect_triangle.restype = C.c_int
        h.or_intersect_triangle.argtypes = [C.POINTER(C.c_float)] * 4 + [C.POINTER(C.c_float)] * 3
        _bind_pixels(h)
        _or = h
    return _or


def _bind_pixels(h):
    h.or_scene_create.restype = C.c_void_p
    h.or_scene_create.argtypes = [C.POINTER(capi.Scene), C.c_int]
    h.or_scene_destroy.argtypes = [C.c_void_p]
    h.or_render_pixels.restype = C.c_int
    h.or_render_pixels.argtypes = [C.c_void_p, C.POINTER(capi.RenderSettings), C.c_void_p, C.c_uint32, C.c_uint32,
                                   C.c_uint32, C.c_void_p, C.c_int]


def oracle_fp64():
    """The double-precision build of the same restatement (ground truth)."""
    global _or64
    if _or64 is None:
        h = _load(ORACLE64_SO)
        _bind_pixels(h)
        _or64 = h
    return _or64


def conv(x, y, width, height, kernel_size):
    """The Accelerator test's convolution (Src/Test/conv.hpp:22-37) of a float32 image x (height x width) with a
    float32 kernel y (kernel_size x kernel_size), accumulated in float in the reference's loop order."""
    import numpy as np

    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    z = np.empty(width * height, np.float32)
    oracle().or_conv(x.ctypes.data, y.ctypes.data, z.ctypes.data, width, height, kernel_size)
    return z


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        sys.path.insert(0, HERE)
        from build_oracle import build_ref as _br

        _br()  # rebuilds a stale library when the reference sources are at hand (PIPER2_REFERENCE), else no-op
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference sources)")
        h = C.CDLL(REF_SO)
        h.ref_scene_create.restype = C.c_void_p
        h.ref_scene_create.argtypes = [C.POINTER(capi.Scene), C.POINTER(capi.RenderSettings), C.c_int]
        h.ref_scene_destroy.argtypes = [C.c_void_p]
        h.ref_render.restype = C.c_int
        h.ref_render.argtypes = [C.c_void_p, C.POINTER(capi.Rect), C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                 C.c_int]
        h.ref_sobol_generate.restype = C.c_float
        h.ref_sobol_generate.argtypes = [C.c_uint64, C.c_uint32]
        h.ref_sobol_start.argtypes = [C.c_uint32] * 4 + [C.POINTER(C.c_uint64), C.POINTER(C.c_float)]
        h.ref_camera_ray.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_float, C.POINTER(C.c_float)]
        _ref = h
    return _ref


class OracleScene:
    """A scene loaded into the oracle (use_bvh for large scenes)."""

    def __init__(self, scene_data, use_bvh=True):
        self.data = scene_data
        self._sc, self._keep = scene_data.to_ctypes()
        self.h = oracle().or_scene_create(C.byref(self._sc), 1 if use_bvh else 0)

    def close(self):
        if self.h:
            oracle().or_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def trace_closest(self, rays, threads=0):
        hits = np.zeros(len(rays), dtype=capi.HIT_DTYPE)
        rays = np.ascontiguousarray(rays)
        oracle().or_trace_closest(self.h, rays.ctypes.data, len(rays), hits.ctypes.data, threads or os.cpu_count())
        return hits

    def trace_any(self, rays, threads=0):
        occ = np.zeros(len(rays), dtype=np.uint32)
        rays = np.ascontiguousarray(rays)
        oracle().or_trace_any(self.h, rays.ctypes.data, len(rays), occ.ctypes.data, threads or os.cpu_count())
        return occ

    def counters(self, rays, closest=True):
        nv, nt = C.c_uint64(), C.c_uint64()
        rays = np.ascontiguousarray(rays)
        oracle().or_trace_counters(self.h, rays.ctypes.data, len(rays), 1 if closest else 0, C.byref(nv), C.byref(nt))
        return nv.value, nt.value

    def bsdf_sample(self, mat, wo, u, front=True):
        """Material `mat`'s BxDF sampled at n (u1, u2) pairs -> (wi (n,3), f (n,3), pdf (n,))."""
        u = np.ascontiguousarray(u, dtype=np.float32)
        n = len(u)
        wo = np.ascontiguousarray(wo, dtype=np.float32)
        wi = np.zeros((n, 3), np.float32)
        f = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        oracle().or_bsdf_sample(self.h, mat, int(front), wo.ctypes.data, n, u.ctypes.data, wi.ctypes.data,
                                f.ctypes.data, pdf.ctypes.data)
        return wi, f, pdf

    def bsdf_eval(self, mat, wo, wi, front=True):
        """Material `mat`'s BxDF value (n,3) and pdf (n,) at directions wi (n,3)."""
        wi = np.ascontiguousarray(wi, dtype=np.float32)
        n = len(wi)
        wo = np.ascontiguousarray(wo, dtype=np.float32)
        f = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        oracle().or_bsdf_eval(self.h, mat, int(front), wo.ctypes.data, n, wi.ctypes.data, f.ctypes.data,
                              pdf.ctypes.data)
        return f, pdf

    def render(self, settings, rect=None, sample_begin=0, sample_count=None, threads=0, samples=True):
        st = settings
        if rect is None:
            rect = full_rect(st)
        if sample_count is None:
            sample_count = st.samples_per_pixel
        film = np.zeros((st.height, st.width, 4), dtype=np.float32)
        out = np.zeros((rect.height, rect.width, sample_count, 5), dtype=np.float32) if samples else None
        rc = oracle().or_render(self.h, C.byref(st), C.byref(rect), sample_begin, sample_count, film.ctypes.data,
                                out.ctypes.data if out is not None else None, threads or os.cpu_count())
        if rc != 0:
            raise RuntimeError(f"or_render failed: {rc}")
        return film, out

    def render_pixels(self, pixels, sample_begin, sample_count, threads=0):
        """Single-precision oracle: resolved RGB of chosen pixels (same accumulation as TruthScene)."""
        return render_pixels(oracle(), self.h, self.data.settings, pixels, sample_begin, sample_count, threads)


def render_pixels(lib, handle, settings, pixels, sample_begin, sample_count, threads=0):
    """Resolved (radiance / weight) RGB of the film pixels `pixels` ((n, 2) x, y) over the given samples."""
    px = np.ascontiguousarray(pixels, dtype=np.uint32)
    out = np.zeros((len(px), 4), dtype=np.float64)
    rc = lib.or_render_pixels(handle, C.byref(settings), px.ctypes.data, len(px), sample_begin, sample_count,
                              out.ctypes.data, threads or os.cpu_count())
    if rc != 0:
        raise RuntimeError(f"or_render_pixels failed: {rc}")
    return out[:, :3] / np.maximum(out[:, 3:4], 1e-300)


class TruthScene:
    """A scene in the double-precision restatement: ground-truth pixel values for relMSE."""

    def __init__(self, scene_data, use_bvh=True):
        self.data = scene_data
        self._sc, self._keep = scene_data.to_ctypes()
        self.h = oracle_fp64().or_scene_create(C.byref(self._sc), 1 if use_bvh else 0)

    def close(self):
        if self.h:
            oracle_fp64().or_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def render_pixels(self, pixels, sample_begin, sample_count, threads=0):
        return render_pixels(oracle_fp64(), self.h, self.data.settings, pixels, sample_begin, sample_count, threads)


class RefScene:
    """A scene loaded into the reference harness (the reference's kernels compiled natively)."""

    def __init__(self, scene_data, use_bvh=True):
        self._sc, self._keep = scene_data.to_ctypes()
        self.settings = scene_data.settings
        self.h = ref().ref_scene_create(C.byref(self._sc), C.byref(self.settings), 1 if use_bvh else 0)

    def close(self):
        if self.h:
            ref().ref_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def render(self, rect=None, sample_begin=0, sample_count=None, threads=0, samples=True):
        st = self.settings
        if rect is None:
            rect = full_rect(st)
        if sample_count is None:
            sample_count = st.samples_per_pixel
        film = np.zeros((st.height, st.width, 4), dtype=np.float32)
        out = np.zeros((rect.height, rect.width, sample_count, 5), dtype=np.float32) if samples else None
        ref().ref_render(self.h, C.byref(rect), sample_begin, sample_count, film.ctypes.data,
                         out.ctypes.data if out is not None else None, threads or os.cpu_count())
        return film, out

    def camera_ray(self, ndc_x, ndc_y, u1, u2):
        o = (C.c_float * 6)()
        ref().ref_camera_ray(self.h, ndc_x, ndc_y, u1, u2, o)
        return np.array(list(o), dtype=np.float32)


def full_rect(settings):
    tr, rc = capi.NDCTransform(), capi.Rect()
    cam = settings.camera
    oracle().or_calc_render_rect(settings.width, settings.height, cam.sensor_size[0] / cam.sensor_size[1],
                                 settings.fit_mode, C.byref(tr), C.byref(rc))
    return rc
