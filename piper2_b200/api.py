"""Python host API over the C ABI, mirroring the reference's tracer interface for this path.

* :class:`Accel`     -- ``Tracer::buildAcceleration`` + the trace queries Embree answers
  (``rtcIntersect1`` / ``rtcOccluded1``, Src/BuiltinComponent/Tracer/Embree/Embree.cpp:267-391), batched.
* :class:`Pipeline`  -- ``Tracer::buildPipeline`` -> ``Pipeline::prepare`` -> ``TraceLauncher::launch``
  (Src/Interface/BuiltinComponent/Tracer.hpp:100-159) and the FixedSampler film resolve
  (Src/BuiltinComponent/RenderDriver/FixedSampler/FixedSampler.cpp:68-133).
* :class:`Batch`     -- many scenes of uneven size rendered through one shared wavefront (no counterpart in
  the reference, which renders one scene per pipeline).
* :class:`Guide`     -- the learned path-guiding network (no counterpart in the reference: its
  PathTracing integrator samples BxDFs only), attached with :meth:`Pipeline.set_guide`.

Device memory and streams come from torch (plumbing only); all compute is in libpiper2_b200.so.
Errors raise :class:`piper2_b200.capi.PB2Error` with the library's message.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise capi.PB2Error("piper2_b200 needs a CUDA device")
    return torch


def _stream():
    torch = _torch()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class Accel:
    """Acceleration structure over a scene's meshes and area-light planes."""

    def __init__(self, scene_data):
        torch = _torch()
        torch.cuda.init()
        self._sc, self._keep = scene_data.to_ctypes()
        h = C.c_void_p()
        capi.check(capi.lib().pb2_accel_create(C.byref(self._sc), _stream(), C.byref(h)))
        self.h = h

    def info(self) -> capi.AccelInfo:
        i = capi.AccelInfo()
        capi.check(capi.lib().pb2_accel_get_info(self.h, C.byref(i)))
        return i

    def validate(self):
        """Structural check of the BVH (raises PB2Error naming the first violation)."""
        capi.check(capi.lib().pb2_accel_validate(self.h))

    def close(self):
        if getattr(self, "h", None):
            capi.lib().pb2_accel_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_counting(self, enable: bool):
        capi.check(capi.lib().pb2_accel_set_counting(self.h, 1 if enable else 0))

    def counters(self):
        nv, nt = C.c_uint64(), C.c_uint64()
        capi.check(capi.lib().pb2_accel_get_counters(self.h, C.byref(nv), C.byref(nt), _stream()))
        return nv.value, nt.value

    # ---- device-pointer calls (torch tensors) ----
    def trace_closest_dev(self, rays_dev, n, hits_dev):
        capi.check(capi.lib().pb2_trace_closest(self.h, C.c_void_p(rays_dev), n, C.c_void_p(hits_dev), _stream()))

    def trace_any_dev(self, rays_dev, n, occ_dev):
        capi.check(capi.lib().pb2_trace_any(self.h, C.c_void_p(rays_dev), n, C.c_void_p(occ_dev), _stream()))

    # ---- host arrays in / out (numpy RAY_DTYPE) ----
    def trace_closest(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=capi.RAY_DTYPE)
        hits = np.zeros(len(rays), dtype=capi.HIT_DTYPE)
        capi.check(capi.lib().pb2_trace_closest_host(self.h, rays.ctypes.data_as(C.c_void_p), len(rays),
                                                     hits.ctypes.data_as(C.c_void_p), _stream()))
        return hits

    def trace_any(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=capi.RAY_DTYPE)
        occ = np.zeros(len(rays), dtype=np.uint32)
        capi.check(capi.lib().pb2_trace_any_host(self.h, rays.ctypes.data_as(C.c_void_p), len(rays),
                                                 occ.ctypes.data_as(C.c_void_p), _stream()))
        return occ


class Builder:
    """The materialized programs of a Piper scene (symbol names and the reference's POD payloads), turned into
    the C ABI's scene and settings by the library (pb2_builder_*).  Host-side only: no GPU is needed."""

    KIND = {"sensor": 0, "integrator": 1, "driver": 2, "sampler": 3, "light_sampler": 4, "surface": 5, "light": 6}

    def __init__(self):
        h = C.c_void_p()
        capi.check(capi.lib().pb2_builder_create(C.byref(h)))
        self.h = h
        self.scene = None
        self.settings = None

    def close(self):
        if getattr(self, "h", None):
            capi.lib().pb2_builder_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _buf(data: bytes):
        b = C.create_string_buffer(bytes(data), max(1, len(data)))
        return b, len(data)

    def register_resource(self, data: bytes) -> int:
        b, n = self._buf(data)
        idx = C.c_uint32()
        capi.check(capi.lib().pb2_builder_register_resource(self.h, b, n, C.byref(idx)))
        return idx.value

    def register_call(self, symbol: str, payload: bytes = b"") -> int:
        b, n = self._buf(payload)
        hd = C.c_uint64()
        capi.check(capi.lib().pb2_builder_register_call(self.h, symbol.encode(), b, n, C.byref(hd)))
        return hd.value

    def add_node(self, traversal: int, translation):
        capi.check(capi.lib().pb2_builder_add_node(self.h, int(traversal), capi.f3(translation)))

    def add_node_transform(self, traversal: int, matrix):
        """A node with a full row-major 3x4 local-to-world transform (scenes.srt_matrix)."""
        m = np.ascontiguousarray(matrix, dtype=np.float32).reshape(12)
        capi.check(capi.lib().pb2_builder_add_node_transform(self.h, int(traversal), m.ctypes.data))

    def add_program(self, kind, symbol: str, payload: bytes = b"") -> int:
        b, n = self._buf(payload)
        idx = C.c_uint32()
        k = self.KIND[kind] if isinstance(kind, str) else int(kind)
        capi.check(capi.lib().pb2_builder_add_program(self.h, k, symbol.encode(), b, n, C.byref(idx)))
        return idx.value

    def add_mesh(self, vertices, indices, material: int, translation=(0.0, 0.0, 0.0), transform=None,
                 texcoords=None):
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        ix = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
        m = capi.Mesh()
        m.vertices, m.indices, m.texcoords = v.ctypes.data, ix.ctypes.data, None
        m.vert_count, m.tri_count, m.material = v.shape[0], ix.shape[0], int(material)
        m.translation[:] = [float(x) for x in translation]
        if transform is not None:
            tr = np.ascontiguousarray(transform, dtype=np.float32).reshape(12)
            m.transform = tr.ctypes.data
        if texcoords is not None:
            tc = np.ascontiguousarray(texcoords, dtype=np.float32).reshape(-1, 2)
            if tc.shape[0] != v.shape[0]:
                raise ValueError("texcoords must hold one (u, v) per vertex")
            m.texcoords = tc.ctypes.data
        capi.check(capi.lib().pb2_builder_add_mesh(self.h, C.byref(m)))  # copied by the library

    def build(self, width: int, height: int, fit_mode: int, samples_per_pixel: int):
        """Fills and returns (capi.Scene, capi.RenderSettings); the scene's arrays live as long as the builder."""
        sc, st = capi.Scene(), capi.RenderSettings()
        capi.check(capi.lib().pb2_builder_build(self.h, width, height, fit_mode, samples_per_pixel, C.byref(sc),
                                                C.byref(st)))
        self.scene, self.settings = sc, st
        return sc, st


class Pipeline:
    """A render pipeline for one scene and one set of render settings."""

    def __init__(self, scene_data, settings=None):
        """scene_data: a scenes.SceneData, or a Builder that has been built (then `settings` defaults to its
        built settings)."""
        torch = _torch()
        torch.cuda.init()
        if isinstance(scene_data, Builder):
            self.settings = settings if settings is not None else scene_data.settings
            self._sc, self._keep = scene_data.scene, scene_data
        else:
            self.settings = settings if settings is not None else scene_data.settings
            self._sc, self._keep = scene_data.to_ctypes()
        h = C.c_void_p()
        capi.check(capi.lib().pb2_pipeline_create(C.byref(self._sc), C.byref(self.settings), _stream(), C.byref(h)))
        self.h = h
        self.rect = capi.Rect()
        self.ndc = capi.NDCTransform()
        capi.check(capi.lib().pb2_pipeline_get_rect(self.h, C.byref(self.rect), C.byref(self.ndc)))

    def close(self):
        if getattr(self, "h", None):
            capi.lib().pb2_pipeline_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def new_film(self):
        torch = _torch()
        return torch.zeros((self.settings.height, self.settings.width, 4), dtype=torch.float32, device="cuda")

    def launch(self, film, rect=None, sample_begin=0, sample_count=None, sample_out=None):
        """TraceLauncher::launch: adds the samples of `rect` to `film` (device tensor H x W x 4)."""
        rect = rect or self.rect
        if sample_count is None:
            sample_count = self.settings.samples_per_pixel
        capi.check(capi.lib().pb2_pipeline_launch(
            self.h, C.byref(rect), sample_begin, sample_count, C.c_void_p(film.data_ptr()),
            C.c_void_p(sample_out.data_ptr()) if sample_out is not None else None, _stream()))

    def render(self, samples=False, rect=None, sample_begin=0, sample_count=None):
        """Full render; returns (film RGBW numpy H x W x 4, per-sample numpy rows x cols x spp x 5 or None)."""
        torch = _torch()
        rect = rect or self.rect
        if sample_count is None:
            sample_count = self.settings.samples_per_pixel
        film = self.new_film()
        out = None
        if samples:
            out = torch.zeros((rect.height, rect.width, sample_count, 5), dtype=torch.float32, device="cuda")
        self.launch(film, rect, sample_begin, sample_count, out)
        torch.cuda.synchronize()
        return film.cpu().numpy(), (out.cpu().numpy() if out is not None else None)

    def set_counting(self, enable: bool):
        """Counting build of the render's traversal queries (rays, node visits, triangle tests per query kind)."""
        capi.check(capi.lib().pb2_pipeline_set_counting(self.h, 1 if enable else 0))

    def trace_counters(self) -> dict:
        """Since counting was switched on: {"extend"|"mis"|"shadow": (rays, node visits, triangle tests)}."""
        c = np.zeros(9, dtype=np.uint64)
        capi.check(capi.lib().pb2_pipeline_get_trace_counters(self.h, c.ctypes.data_as(C.c_void_p), _stream()))
        return {k: tuple(int(x) for x in c[3 * i:3 * i + 3]) for i, k in enumerate(("extend", "mis", "shadow"))}

    def set_path_slots(self, slots: int):
        """Bound the path slots in flight; a larger launch refills freed slots with its remaining paths."""
        capi.check(capi.lib().pb2_pipeline_set_path_slots(self.h, int(slots)))

    def set_graphs(self, enable: bool):
        """Run the bounce loop of later launches as CUDA graphs (the default) or as plain launches."""
        capi.check(capi.lib().pb2_pipeline_set_graphs(self.h, 1 if enable else 0))

    def resolve(self, film):
        torch = _torch()
        rgb = torch.empty((self.settings.height, self.settings.width, 3), dtype=torch.float32, device="cuda")
        capi.check(capi.lib().pb2_film_resolve(C.c_void_p(film.data_ptr()), self.settings.width * self.settings.height,
                                               C.c_void_p(rgb.data_ptr()), _stream()))
        return rgb

    def camera_rays(self, sample=0, rect=None):
        torch = _torch()
        rect = rect or self.rect
        n = rect.width * rect.height
        rays = torch.empty((n, 8), dtype=torch.float32, device="cuda")
        pts = torch.empty((n, 2), dtype=torch.float32, device="cuda")
        capi.check(capi.lib().pb2_pipeline_camera_rays(self.h, C.byref(rect), sample, C.c_void_p(rays.data_ptr()),
                                                       C.c_void_p(pts.data_ptr()), _stream()))
        torch.cuda.synchronize()
        return rays.cpu().numpy(), pts.cpu().numpy()

    def stats(self) -> capi.LaunchStats:
        s = capi.LaunchStats()
        capi.check(capi.lib().pb2_pipeline_get_stats(self.h, C.byref(s), _stream()))
        return s

    def set_guide(self, guide, selection_prob=0.5, record_capacity=1 << 20, weight_quantile=0.99, spatial_cells=0,
                  guided_types=0, max_guided_depth=0):
        """Attach a :class:`Guide` (None detaches); later launches sample and record with it."""
        self._guide = guide
        if guide is None:
            capi.check(capi.lib().pb2_pipeline_set_guide(self.h, None, None))
            return
        st = capi.GuideSettings(float(selection_prob), int(record_capacity), float(weight_quantile), int(spatial_cells),
                                int(guided_types), int(max_guided_depth))
        capi.check(capi.lib().pb2_pipeline_set_guide(self.h, guide.h, C.byref(st)))

    def train_guide(self, steps, batch=1 << 16, learning_rate=1e-2) -> float:
        """Adam steps on the records of the launches since the last call; returns the last loss."""
        loss = C.c_float(0.0)
        capi.check(capi.lib().pb2_pipeline_train_guide(self.h, steps, batch, learning_rate, C.byref(loss), _stream()))
        return loss.value

    def render_guided(self, film, spp, spp_per_pass=4, train_steps=4, batch=1 << 16, learning_rate=1e-2,
                      train_passes=None, rect=None, sample_begin=0):
        """Progressive guided render: `spp / spp_per_pass` launches into `film`, each followed (for the first
        `train_passes`, default all) by `train_steps` Adam steps on the records it produced.  Every pass is
        an unbiased estimate, so the film averages all of them.  Returns the losses."""
        losses = []
        passes = max(1, spp // spp_per_pass)
        for p in range(passes):
            self.launch(film, rect, sample_begin + p * spp_per_pass, spp_per_pass)
            if train_steps and (train_passes is None or p < train_passes) and p + 1 < passes:
                losses.append(self.train_guide(train_steps, batch, learning_rate))
        return losses


class _DeviceArray:
    """A float32 device buffer owned by the library, seen by torch through the CUDA array interface."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4", "data": (ptr, False), "version": 3}


class Batch:
    """Scenes rendered together: one wavefront of path slots refilled from all scenes' (pixel, sample) space."""

    def __init__(self, scene_datas, settings=None):
        torch = _torch()
        torch.cuda.init()
        self.scene_datas = list(scene_datas)
        n = len(self.scene_datas)
        self._conv = [sd.to_ctypes() for sd in self.scene_datas]
        self._scenes = (capi.Scene * n)(*[c[0] for c in self._conv])
        sts = settings if settings is not None else [sd.settings for sd in self.scene_datas]
        self._settings = (capi.RenderSettings * n)(*sts)
        h = C.c_void_p()
        capi.check(capi.lib().pb2_batch_create(C.cast(self._scenes, C.c_void_p), C.cast(self._settings, C.c_void_p),
                                               n, _stream(), C.byref(h)))
        self.h = h
        self.count = n

    def close(self):
        if getattr(self, "h", None):
            capi.lib().pb2_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def config(self) -> capi.BatchConfig:
        c = capi.BatchConfig()
        capi.check(capi.lib().pb2_batch_get_config(self.h, C.byref(c)))
        return c

    def set_config(self, **kw):
        c = self.config
        for k, v in kw.items():
            setattr(c, k, int(v))
        capi.check(capi.lib().pb2_batch_set_config(self.h, C.byref(c)))

    def autotune(self):
        """Picks capacity and launch shapes by timing short runs; returns (config, tuning ms)."""
        c = capi.BatchConfig()
        ms = C.c_float(0.0)
        capi.check(capi.lib().pb2_batch_autotune(self.h, _stream(), C.byref(c), C.byref(ms)))
        return c, ms.value

    def render(self):
        capi.check(capi.lib().pb2_batch_render(self.h, _stream()))

    def film(self, i):
        """Scene i's RGBW film as a numpy array (H x W x 4)."""
        torch = _torch()
        ptr = C.c_void_p()
        w, h = C.c_uint32(), C.c_uint32()
        capi.check(capi.lib().pb2_batch_film(self.h, i, C.byref(ptr), C.byref(w), C.byref(h)))
        view = torch.as_tensor(_DeviceArray(ptr.value, (h.value, w.value, 4)), device="cuda")
        torch.cuda.synchronize()
        return view.cpu().numpy()

    def timing(self):
        """(per-scene completion ms, total device ms, wavefront iterations) of the last render."""
        ms = np.zeros(self.count, dtype=np.float32)
        tot = C.c_float(0.0)
        it = C.c_uint32(0)
        capi.check(capi.lib().pb2_batch_timing(self.h, ms.ctypes.data_as(C.c_void_p), self.count, C.byref(tot),
                                               C.byref(it)))
        return ms, tot.value, it.value

    def stats(self) -> capi.LaunchStats:
        s = capi.LaunchStats()
        capi.check(capi.lib().pb2_batch_get_stats(self.h, C.byref(s)))
        return s


class Guide:
    """Path-guiding MLP (96-64-64-64-64-48, 8 von Mises-Fisher lobes) with Adam state on the device."""

    def __init__(self, seed=1):
        _torch().cuda.init()
        h = C.c_void_p()
        capi.check(capi.lib().pb2_guide_create(seed, C.byref(h)))
        self.h = h

    @staticmethod
    def param_count() -> int:
        return int(capi.lib().pb2_guide_param_count())

    def close(self):
        if getattr(self, "h", None):
            capi.lib().pb2_guide_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_gradient_hook(self, fn):
        """Call fn(grad) with each training step's gradient (a float32 CUDA tensor of param_count() values on
        the library's memory, to be modified in place, e.g. all-reduced over ranks) before the Adam update.
        fn runs on the training call's thread with torch's current stream; None removes the hook."""
        if fn is None:
            capi.check(capi.lib().pb2_guide_set_gradient_hook(self.h, None, None))
            self._hook = None
            return
        torch = _torch()

        def _call(ptr, count, stream, user):
            try:
                grad = torch.as_tensor(_DeviceArray(ptr, (count,)), device="cuda")
                fn(grad)
                return 0
            except Exception:  # reported to the library as a failed step
                return capi.PB2_ERR_INVALID_ARGUMENT

        self._hook = capi.GRADIENT_HOOK(_call)  # kept alive as long as the guide
        capi.check(capi.lib().pb2_guide_set_gradient_hook(self.h, C.cast(self._hook, C.c_void_p), None))

    def get_params(self) -> np.ndarray:
        out = np.empty(self.param_count(), dtype=np.float32)
        capi.check(capi.lib().pb2_guide_get_params(self.h, out.ctypes.data_as(C.c_void_p), len(out)))
        return out

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        capi.check(capi.lib().pb2_guide_set_params(self.h, p.ctypes.data_as(C.c_void_p), len(p)))

    def forward(self, features: np.ndarray, tiles: str = "tcgen05") -> np.ndarray:
        """features (n, 12) -> raw outputs (n, 48); tiles = "tcgen05" (default) or "mma" (mma.sync)."""
        torch = _torch()
        f = torch.from_numpy(np.ascontiguousarray(features, dtype=np.float32)).cuda()
        n = f.shape[0]
        out = torch.empty((n, 48), dtype=torch.float32, device="cuda")
        fn = capi.lib().pb2_guide_forward if tiles == "tcgen05" else capi.lib().pb2_guide_forward_mma
        capi.check(fn(self.h, C.c_void_p(f.data_ptr()), n, C.c_void_p(out.data_ptr()), _stream()))
        torch.cuda.synchronize()
        return out.cpu().numpy()

    def gradient(self, records: np.ndarray, tiles: str = "tcgen05"):
        """records (n, 16) -> (gradient over the flat parameters, loss); tiles = "tcgen05" (default, the
        training kernel) or "mma" (the mma.sync cross-check)."""
        torch = _torch()
        r = torch.from_numpy(np.ascontiguousarray(records, dtype=np.float32)).cuda()
        g = np.empty(self.param_count(), dtype=np.float32)
        loss = C.c_float(0.0)
        fn = capi.lib().pb2_guide_gradient if tiles == "tcgen05" else capi.lib().pb2_guide_gradient_mma
        capi.check(fn(self.h, C.c_void_p(r.data_ptr()), r.shape[0], g.ctypes.data_as(C.c_void_p), C.byref(loss),
                      _stream()))
        return g, loss.value

    def train(self, records, learning_rate=5e-3) -> float:
        """One Adam step on a batch; `records` is a (n, 16) numpy array or float32 CUDA tensor."""
        torch = _torch()
        r = records if isinstance(records, torch.Tensor) else torch.from_numpy(
            np.ascontiguousarray(records, dtype=np.float32)).cuda()
        loss = C.c_float(0.0)
        capi.check(capi.lib().pb2_guide_train(self.h, C.c_void_p(r.data_ptr()), r.shape[0], learning_rate,
                                              C.byref(loss), _stream()))
        return loss.value


def sobol_generate(index: np.ndarray, dim: np.ndarray) -> np.ndarray:
    torch = _torch()
    idx = torch.from_numpy(np.ascontiguousarray(index, dtype=np.uint64).view(np.int64)).cuda()
    dm = torch.from_numpy(np.ascontiguousarray(dim, dtype=np.uint32).view(np.int32)).cuda()
    out = torch.empty(len(index), dtype=torch.float32, device="cuda")
    capi.check(capi.lib().pb2_sobol_generate(C.c_void_p(idx.data_ptr()), C.c_void_p(dm.data_ptr()), len(index),
                                             C.c_void_p(out.data_ptr()), _stream()))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def sobol_start(log2res: int, pixel_sample: np.ndarray):
    torch = _torch()
    ps = torch.from_numpy(np.ascontiguousarray(pixel_sample, dtype=np.uint32).view(np.int32).reshape(-1)).cuda()
    n = len(pixel_sample)
    idx = torch.empty(n, dtype=torch.int64, device="cuda")
    off = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    capi.check(capi.lib().pb2_sobol_start(log2res, C.c_void_p(ps.data_ptr()), n, C.c_void_p(idx.data_ptr()),
                                          C.c_void_p(off.data_ptr()), _stream()))
    torch.cuda.synchronize()
    return idx.cpu().numpy().view(np.uint64), off.cpu().numpy()
