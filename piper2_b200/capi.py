"""ctypes mirror of include/piper2_b200.h and the loader of the CUDA library.

The library is the product: ``piper2_b200/_lib/libpiper2_b200.so`` built by ``piper2_b200.build``.
There is no fallback -- if it is missing, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpiper2_b200.so")

PB2_OK = 0
PB2_ERR_INVALID_ARGUMENT = 1
PB2_ERR_CUDA = 2
PB2_ERR_OUT_OF_MEMORY = 3
PB2_ERR_NOT_SUPPORTED = 4
PB2_ERR_DEVICE_TIMEOUT = 5
PB2_ERR_QUEUE_OVERFLOW = 6
PB2_INVALID_PRIM = 0xFFFFFFFF
PB2_PLANE_FLAG = 0x80000000

SURFACE = {"BlackBody": 0, "Matte": 1, "Plastic": 2, "Glass": 3, "Mirror": 4, "Substrate": 5, "Conductor": 6}
FILTER = {"box": 0, "triangle": 1, "gaussian": 2}
FIT = {"Fill": 0, "OverScan": 1}


class Ray(C.Structure):
    _fields_ = [("org", C.c_float * 3), ("tmin", C.c_float), ("dir", C.c_float * 3), ("tmax", C.c_float)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("prim", C.c_uint32), ("u", C.c_float), ("v", C.c_float)]


RAY_DTYPE = np.dtype([("org", "<f4", 3), ("tmin", "<f4"), ("dir", "<f4", 3), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("prim", "<u4"), ("u", "<f4"), ("v", "<f4")])
assert RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 16


class Mesh(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("indices", C.c_void_p), ("texcoords", C.c_void_p),
                ("vert_count", C.c_uint32), ("tri_count", C.c_uint32), ("material", C.c_uint32),
                ("translation", C.c_float * 3), ("transform", C.c_void_p)]


class SRT(C.Structure):
    """pb2_srt: the reference's TransformSRT (Src/Kernel/Transform.hpp:390-393)."""
    _fields_ = [("scale", C.c_float * 3), ("skew", C.c_float * 3), ("shift", C.c_float * 3), ("quat", C.c_float * 4),
                ("translation", C.c_float * 3)]


class Plane(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("u", C.c_float * 3), ("v", C.c_float * 3), ("normal", C.c_float * 3),
                ("tangent", C.c_float * 3), ("max_det_comp", C.c_uint32)]


class AreaLight(C.Structure):
    _fields_ = [("radiance", C.c_float * 3), ("first_plane", C.c_uint32), ("plane_count", C.c_uint32),
                ("translation", C.c_float * 3)]


class Material(C.Structure):
    _fields_ = [("type", C.c_uint32), ("color0", C.c_float * 4), ("color1", C.c_float * 4),
                ("roughness", C.c_float * 2), ("texture", C.c_uint32 * 4)]


class Texture(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("channel", C.c_uint32), ("wrap", C.c_uint32), ("width", C.c_uint32),
                ("height", C.c_uint32), ("texels", C.c_void_p), ("scale", C.c_float), ("black", C.c_float * 4),
                ("white", C.c_float * 4)]


TEXTURE_CHECKERBOARD, TEXTURE_IMAGE = 1, 2
WRAP = {"Repeat": 0, "Mirror": 1}


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3),
                ("sensor_size", C.c_float * 2), ("focal_length", C.c_float), ("aperture_radius", C.c_float)]


class Scene(C.Structure):
    _fields_ = [("meshes", C.POINTER(Mesh)), ("mesh_count", C.c_uint32), ("planes", C.POINTER(Plane)),
                ("plane_count", C.c_uint32), ("area_lights", C.POINTER(AreaLight)), ("area_light_count", C.c_uint32),
                ("materials", C.POINTER(Material)), ("material_count", C.c_uint32),
                ("env_radiance", C.c_float * 3), ("textures", C.POINTER(Texture)), ("texture_count", C.c_uint32)]


class RenderSettings(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("fit_mode", C.c_uint32),
                ("samples_per_pixel", C.c_uint32), ("scramble", C.c_uint32), ("max_depth", C.c_uint32),
                ("min_rr_depth", C.c_uint32), ("filter", C.c_uint32), ("gaussian_alpha", C.c_float),
                ("camera", Camera), ("scramble_seed", C.c_uint32)]


class Rect(C.Structure):
    _fields_ = [("left", C.c_uint32), ("top", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32)]


class NDCTransform(C.Structure):
    _fields_ = [("ox", C.c_float), ("oy", C.c_float), ("sx", C.c_float), ("sy", C.c_float)]


class AccelInfo(C.Structure):
    _fields_ = [("triangle_count", C.c_uint32), ("node_count", C.c_uint32), ("leaf_triangle_slots", C.c_uint32),
                ("plane_count", C.c_uint32), ("device_bytes", C.c_uint64), ("build_ms", C.c_float)]


class LaunchStats(C.Structure):
    _fields_ = [("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("paths", C.c_uint64),
                ("path_vertices", C.c_uint64), ("depth_histogram", C.c_uint32 * 32)]


assert C.sizeof(Plane) == 64 and C.sizeof(Material) == 60


class PB2Error(RuntimeError):
    pass


_lib = None

# (name, restype, argtypes) for every entry point declared in include/piper2_b200.h
class BatchConfig(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("shade_block", C.c_uint32), ("trace_blocks_per_sm", C.c_uint32),
                ("use_graph", C.c_uint32)]


class GuideSettings(C.Structure):
    _fields_ = [("selection_prob", C.c_float), ("record_capacity", C.c_uint32), ("weight_quantile", C.c_float),
                ("spatial_cells", C.c_uint32), ("guided_types", C.c_uint32),
                ("max_guided_depth", C.c_uint32)]


SIGNATURES = [
    ("pb2_last_error", C.c_char_p, []),
    ("pb2_abi_version", C.c_int, []),
    ("pb2_set_device", C.c_int, [C.c_int]),
    ("pb2_plane_make", C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(Plane)]),
    ("pb2_srt_matrix", C.c_int, [C.POINTER(SRT), C.POINTER(C.c_float)]),
    ("pb2_plane_transform", C.c_int, [C.POINTER(Plane), C.POINTER(C.c_float), C.POINTER(Plane)]),
    ("pb2_camera_from_config", C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                          C.POINTER(C.c_float), C.c_float, C.c_float, C.POINTER(Camera)]),
    ("pb2_calc_render_rect", C.c_int, [C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, C.POINTER(NDCTransform),
                                        C.POINTER(Rect)]),
    ("pb2_sobol_generate", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pb2_sobol_start", C.c_int, [C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pb2_sobol_table_digest", C.c_char_p, []),
    ("pb2_accel_create", C.c_int, [C.POINTER(Scene), C.c_void_p, C.POINTER(C.c_void_p)]),
    ("pb2_accel_destroy", C.c_int, [C.c_void_p]),
    ("pb2_accel_get_info", C.c_int, [C.c_void_p, C.POINTER(AccelInfo)]),
    ("pb2_accel_validate", C.c_int, [C.c_void_p]),
    ("pb2_trace_closest", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pb2_trace_any", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pb2_trace_closest_host", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pb2_trace_any_host", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pb2_trace_closest_nalloc", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pb2_accel_set_counting", C.c_int, [C.c_void_p, C.c_int]),
    ("pb2_accel_get_counters", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_void_p]),
    ("pb2_pipeline_create", C.c_int, [C.POINTER(Scene), C.POINTER(RenderSettings), C.c_void_p,
                                       C.POINTER(C.c_void_p)]),
    ("pb2_pipeline_destroy", C.c_int, [C.c_void_p]),
    ("pb2_pipeline_get_rect", C.c_int, [C.c_void_p, C.POINTER(Rect), C.POINTER(NDCTransform)]),
    ("pb2_pipeline_launch", C.c_int, [C.c_void_p, C.POINTER(Rect), C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    ("pb2_film_resolve", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pb2_pipeline_get_stats", C.c_int, [C.c_void_p, C.POINTER(LaunchStats), C.c_void_p]),
    ("pb2_pipeline_camera_rays", C.c_int, [C.c_void_p, C.POINTER(Rect), C.c_uint32, C.c_void_p, C.c_void_p,
                                            C.c_void_p]),
    ("pb2_batch_create", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_void_p)]),
    ("pb2_batch_destroy", C.c_int, [C.c_void_p]),
    ("pb2_batch_get_config", C.c_int, [C.c_void_p, C.POINTER(BatchConfig)]),
    ("pb2_batch_set_config", C.c_int, [C.c_void_p, C.POINTER(BatchConfig)]),
    ("pb2_batch_autotune", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(BatchConfig), C.POINTER(C.c_float)]),
    ("pb2_batch_render", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pb2_batch_film", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint32)]),
    ("pb2_batch_timing", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_uint32)]),
    ("pb2_batch_get_stats", C.c_int, [C.c_void_p, C.POINTER(LaunchStats)]),
    ("pb2_guide_param_count", C.c_uint32, []),
    ("pb2_guide_create", C.c_int, [C.c_uint32, C.POINTER(C.c_void_p)]),
    ("pb2_guide_destroy", C.c_int, [C.c_void_p]),
    ("pb2_guide_set_params", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    ("pb2_guide_get_params", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    ("pb2_guide_forward", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pb2_guide_forward_async", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pb2_guide_forward_mma", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pb2_guide_gradient", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_float),
                                      C.c_void_p]),
    ("pb2_guide_train", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.POINTER(C.c_float), C.c_void_p]),
    ("pb2_guide_gradient_mma", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_float),
                                          C.c_void_p]),
    ("pb2_guide_set_gradient_hook", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pb2_pipeline_set_guide", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(GuideSettings)]),
    ("pb2_pipeline_set_path_slots", C.c_int, [C.c_void_p, C.c_uint32]),
    ("pb2_pipeline_set_graphs", C.c_int, [C.c_void_p, C.c_int]),
    ("pb2_pipeline_set_counting", C.c_int, [C.c_void_p, C.c_int]),
    ("pb2_pipeline_get_trace_counters", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pb2_pipeline_set_guide_dump", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("pb2_builder_create", C.c_int, [C.POINTER(C.c_void_p)]),
    ("pb2_builder_destroy", C.c_int, [C.c_void_p]),
    ("pb2_builder_register_resource", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint32)]),
    ("pb2_builder_register_call", C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint64)]),
    ("pb2_builder_add_node", C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p]),
    ("pb2_builder_add_node_transform", C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p]),
    ("pb2_builder_add_program", C.c_int, [C.c_void_p, C.c_uint32, C.c_char_p, C.c_void_p, C.c_size_t,
                                          C.POINTER(C.c_uint32)]),
    ("pb2_builder_add_mesh", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pb2_builder_build", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                    C.c_void_p]),
    ("pb2_pipeline_train_guide", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.POINTER(C.c_float),
                                            C.c_void_p]),
    # accelerator (Accelerator.hpp:130-161)
    ("pb2_acc_create", C.c_int, [C.c_uint32, C.POINTER(C.c_void_p)]),
    ("pb2_acc_destroy", C.c_int, [C.c_void_p]),
    ("pb2_acc_native_platform", C.c_char_p, [C.c_void_p]),
    ("pb2_acc_get_info", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_uint32)]),
    ("pb2_acc_create_buffer", C.c_int, [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_void_p)]),
    ("pb2_acc_create_tiled_output", C.c_int, [C.c_void_p, C.c_size_t, C.c_size_t, C.POINTER(C.c_void_p)]),
    ("pb2_acc_create_resource_lut", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_uint32, C.POINTER(C.c_void_p)]),
    ("pb2_resource_get_handle", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("pb2_resource_release", C.c_int, [C.c_void_p]),
    ("pb2_tiled_output_mark_dirty", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pb2_tiled_output_download", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    ("pb2_acc_compile_kernel", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    ("pb2_acc_register_kernel", C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p]),
    ("pb2_kernel_release", C.c_int, [C.c_void_p]),
    ("pb2_acc_launch_kernel", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(C.c_void_p)]),
    ("pb2_acc_pack_launch", C.c_int, [C.POINTER(C.c_uint64), C.c_uint32, C.c_void_p, C.POINTER(C.c_uint32), C.c_uint32,
                                      C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    ("pb2_future_wait", C.c_int, [C.c_void_p]),
    ("pb2_future_ready", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("pb2_future_release", C.c_int, [C.c_void_p]),
]

# void (*)(void* dst, size_t size, void* user): fills a buffer's initial bytes (pb2_acc_create_buffer)
FILL_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_size_t, C.c_void_p)


# int (*)(float* grad_dev, uint32_t count, void* stream, void* user)
GRADIENT_HOOK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p)


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PB2Error(f"{LIB_PATH} is missing: run `python -c 'import __graft_entry__ as g; g.build()'`")
        h = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


def check(code: int) -> None:
    if code != PB2_OK:
        msg = lib().pb2_last_error()
        raise PB2Error(f"piper2_b200 error {code}: {msg.decode() if msg else ''}")


def f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])
