"""The C-ABI library loads on a machine without a GPU, exports every entry point include/piper2_b200.h
declares, and its host-only helpers agree with the oracle's restatements."""
import ctypes as C
import os
import re

import numpy as np

from piper2_b200 import capi, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "piper2_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\s*\*)\s*(pb2_[a-z0-9_]+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = capi.lib()
    names = _declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert lib.pb2_abi_version() == 1
    assert {s[0] for s in capi.SIGNATURES} >= set(names)


def test_sobol_digest_compiled_in(oracle):
    assert capi.lib().pb2_sobol_table_digest() == oracle.oracle().or_sobol_digest()


def test_plane_make_matches_oracle(oracle):
    f = lambda t: (C.c_float * 3)(*t)  # noqa: E731
    for origin, u, v in [((0.375, 0.999, 0.375), (0.25, 0, 0), (0, 0, 0.25)), ((1, 2, 3), (0.3, -0.2, 0.7), (0.1, 0.9, -0.4))]:
        a, b = capi.Plane(), capi.Plane()
        capi.check(capi.lib().pb2_plane_make(f(origin), f(u), f(v), C.byref(a)))
        oracle.oracle().or_plane_make(f(origin), f(u), f(v), C.byref(b))
        assert bytes(a) == bytes(b)


def test_camera_and_render_rect(oracle):
    cam = capi.Camera()
    capi.check(capi.lib().pb2_camera_from_config(capi.f3((0.5, 0.5, -1.4)), capi.f3((0.5, 0.5, 0.5)),
                                                 capi.f3((0, 2, 0)), (C.c_float * 2)(36.0, 24.0), 35.0, 8.0,
                                                 C.byref(cam)))
    py = scenes.camera_from_config((0.5, 0.5, -1.4), (0.5, 0.5, 0.5), (0, 2, 0), (36.0, 24.0), 35.0, 8.0)
    assert bytes(cam) == bytes(py)
    for w, h, aspect, fit in [(1920, 1080, 1.5, 0), (1920, 1080, 1.5, 1), (256, 256, 1.0, 0), (640, 480, 2.0, 1),
                              (480, 640, 1.0, 1)]:
        t1, r1, t2, r2 = capi.NDCTransform(), capi.Rect(), capi.NDCTransform(), capi.Rect()
        capi.check(capi.lib().pb2_calc_render_rect(w, h, aspect, fit, C.byref(t1), C.byref(r1)))
        oracle.oracle().or_calc_render_rect(w, h, aspect, fit, C.byref(t2), C.byref(r2))
        assert bytes(t1) == bytes(t2) and bytes(r1) == bytes(r2)


def test_errors_without_gpu():
    lib = capi.lib()
    assert lib.pb2_plane_make(None, None, None, None) == 1
    assert b"null" in lib.pb2_last_error()
    assert lib.pb2_calc_render_rect(0, 0, 1.0, 0, None, None) == 1


def test_scene_generators_deterministic():
    a = scenes.cornell_box(seed=3)
    b = scenes.cornell_box(seed=3)
    assert all(np.array_equal(x.vertices, y.vertices) for x, y in zip(a.meshes, b.meshes))
    assert a.triangle_count == 34
    s = scenes.triangle_soup(1000, seed=1)
    assert s.triangle_count == 1000
    r = scenes.soup_rays(100, seed=1)
    assert np.allclose(np.linalg.norm(r["dir"], axis=1), 1, atol=1e-6)


def test_ctypes_structs_match_the_header(tmp_path):
    """Every struct the Python binding mirrors has the header's size and field offsets (a C probe compiled
    with gcc against include/piper2_b200.h prints them)."""
    import subprocess

    pairs = {"Ray": "pb2_ray", "Hit": "pb2_hit", "Mesh": "pb2_mesh", "Plane": "pb2_plane",
             "AreaLight": "pb2_area_light", "Material": "pb2_material", "Camera": "pb2_camera", "Scene": "pb2_scene",
             "RenderSettings": "pb2_render_settings", "Rect": "pb2_rect", "NDCTransform": "pb2_ndc_transform",
             "AccelInfo": "pb2_accel_info", "LaunchStats": "pb2_launch_stats", "BatchConfig": "pb2_batch_config",
             "GuideSettings": "pb2_guide_settings", "SRT": "pb2_srt", "Texture": "pb2_texture"}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "piper2_b200.h"', "int main(void) {"]
    for py, c in pairs.items():
        cls = getattr(capi, py)
        lines.append(f'    printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in cls._fields_:
            lines.append(f'    printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines.append("    return 0;\n}")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run(["gcc", "-std=c11", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for py in pairs:
        cls = getattr(capi, py)
        assert got[(py, "size")] == C.sizeof(cls), py
        for name, _ in cls._fields_:
            assert got[(py, name)] == getattr(cls, name).offset, (py, name)
