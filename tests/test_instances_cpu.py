"""Instance transforms (the reference's TransformSRT, Src/Kernel/Transform.hpp:390-393, handed to Embree as an
RTCQuaternionDecomposition, Tracer/Embree/Embree.cpp:699-703): the SRT -> matrix helper against a float64 restatement
of local-to-world = T * R * S, the plane mapping, and the flattening of transformed instances -- the oracle's scene
with a transformed mesh traces exactly like the same mesh with its vertices transformed beforehand.  Host-side
only: runs without a GPU."""
import math

import numpy as np
import pytest

from piper2_b200 import capi, scenes

f32 = np.float32


def _matrix64(scale, skew, shift, quat, trans):
    w, x, y, z = np.asarray(quat, np.float64) / np.linalg.norm(quat)
    r = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                  [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                  [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
    s = np.array([[scale[0], skew[0], skew[1], shift[0]], [0, scale[1], skew[2], shift[1]],
                  [0, 0, scale[2], shift[2]], [0, 0, 0, 1]], np.float64)
    t = np.eye(4)
    t[:3, :3] = r
    t[:3, 3] = trans
    return (t @ s)[:3]


def test_srt_matrix_is_t_r_s():
    rng = np.random.default_rng(0)
    for _ in range(200):
        scale, skew, shift = rng.uniform(0.2, 3, 3), rng.uniform(-0.5, 0.5, 3), rng.uniform(-1, 1, 3)
        quat, trans = rng.normal(size=4), rng.uniform(-5, 5, 3)
        m = scenes.srt_matrix(translation=trans, scale=scale, quat=quat, skew=skew, shift=shift).reshape(3, 4)
        exp = _matrix64(scale, skew, shift, quat, trans)
        np.testing.assert_allclose(m, exp, rtol=0, atol=2e-5 * (1 + np.abs(exp).max()))


def test_srt_identity_and_translation_are_exact():
    m = scenes.srt_matrix()
    assert np.array_equal(m, np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], f32))
    m = scenes.srt_matrix(translation=(0.25, -3.5, 7.0))
    assert np.array_equal(m, np.array([1, 0, 0, 0.25, 0, 1, 0, -3.5, 0, 0, 1, 7.0], f32))


def test_srt_rotation_is_orthonormal_and_normalises_the_quaternion():
    rng = np.random.default_rng(1)
    for _ in range(50):
        q = rng.normal(size=4)
        a = scenes.srt_matrix(quat=q).reshape(3, 4)[:, :3].astype(np.float64)
        b = scenes.srt_matrix(quat=3.0 * q).reshape(3, 4)[:, :3].astype(np.float64)
        np.testing.assert_allclose(a @ a.T, np.eye(3), atol=1e-6)
        assert abs(np.linalg.det(a) - 1) < 1e-5
        np.testing.assert_allclose(a, b, atol=1e-6)


def test_euler_quaternion_follows_the_reference_formula():
    """PiperRenderer.cpp:113-124: the half angles of (pitch, yaw, roll) combined as written there."""
    rng = np.random.default_rng(2)
    for p, y, r in rng.uniform(-math.pi, math.pi, (50, 3)):
        q = scenes.euler_quaternion(p, y, r)
        cp, sp, cy, sy, cr, sr = (math.cos(p / 2), math.sin(p / 2), math.cos(y / 2), math.sin(y / 2),
                                  math.cos(r / 2), math.sin(r / 2))
        exp = (cr * cp * cy + sr * sp * sy, cr * sp * cy + sr * cp * sy, cr * cp * sy - sr * sp * cy,
               sr * cp * cy - cr * sp * sy)
        np.testing.assert_allclose(q, exp, atol=1e-6)
        assert abs(np.linalg.norm(q) - 1) < 1e-6


def test_srt_matrix_rejects_bad_input():
    import ctypes as C

    lib = capi.lib()
    out = (C.c_float * 12)()
    t = scenes.srt(quat=(0, 0, 0, 0))
    assert lib.pb2_srt_matrix(C.byref(t), out) == capi.PB2_ERR_INVALID_ARGUMENT
    t = scenes.srt(scale=(1, float("nan"), 1))
    assert lib.pb2_srt_matrix(C.byref(t), out) == capi.PB2_ERR_INVALID_ARGUMENT
    assert lib.pb2_srt_matrix(None, out) == capi.PB2_ERR_INVALID_ARGUMENT


def test_plane_transform_maps_the_parallelogram():
    rng = np.random.default_rng(3)
    pl = scenes.plane_make((0.1, 0.2, 0.3), (0.5, 0.0, 0.1), (0.0, 0.3, 0.2))
    for _ in range(20):
        m = scenes.srt_matrix(translation=rng.uniform(-1, 1, 3), scale=rng.uniform(0.5, 2, 3), quat=rng.normal(size=4))
        out = scenes.plane_transform(pl, m)
        mm = m.reshape(3, 4).astype(np.float64)
        np.testing.assert_allclose(out.origin, mm[:, :3] @ np.array(pl.origin) + mm[:, 3], atol=1e-5)
        np.testing.assert_allclose(out.u, mm[:, :3] @ np.array(pl.u), atol=1e-5)
        np.testing.assert_allclose(out.v, mm[:, :3] @ np.array(pl.v), atol=1e-5)
        n = np.linalg.inv(mm[:, :3]).T @ np.array(pl.normal)
        np.testing.assert_allclose(out.normal, n / np.linalg.norm(n), atol=1e-5)


def _bake(mesh):
    """The instance's vertices in world space with the library's operation order, in float32."""
    v = mesh.vertices.astype(f32)
    if mesh.transform is None:
        return v + np.asarray(mesh.translation, f32)
    m = np.asarray(mesh.transform, f32).reshape(3, 4)
    out = ((m[:, 0] * v[:, :1] + m[:, 1] * v[:, 1:2]) + m[:, 2] * v[:, 2:3]) + m[:, 3]
    return out + np.asarray(mesh.translation, f32)


def test_oracle_flattens_transformed_instances_exactly(oracle):
    sd = scenes.instanced_room(seed=4)
    baked = scenes.instanced_room(seed=4)
    for m in baked.meshes:
        m.vertices, m.transform, m.translation = _bake(m), None, (0.0, 0.0, 0.0)
    rng = np.random.default_rng(5)
    n = 4096
    rays = np.zeros(n, capi.RAY_DTYPE)
    rays["org"] = rng.uniform(0.05, 0.95, (n, 3))
    d = rng.normal(size=(n, 3))
    rays["dir"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays["tmax"] = 1e30
    a = oracle.OracleScene(sd, use_bvh=True).trace_closest(rays)
    b = oracle.OracleScene(baked, use_bvh=True).trace_closest(rays)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert (a["prim"] >= 10).sum() > 100  # the instanced boxes are hit


def test_builder_maps_lights_and_copies_transforms():
    """Component programs as the Piper tracer delivers them (the payload fixture), with the light's and the
    camera's nodes given full transforms: the light's planes arrive mapped into world space (translation 0), the
    camera stands at its node's origin, and a mesh keeps its instance matrix."""
    import json
    import os

    from piper2_b200 import api

    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "payloads.json")) as f:
        steps = json.load(f)["cornell_box"]
    light_m = scenes.srt_matrix(translation=(0.1, -0.05, 0.0), quat=scenes.euler_quaternion(0.3, 0.0, 0.2))
    cam_m = scenes.srt_matrix(translation=(0.5, 0.5, -1.4), quat=scenes.euler_quaternion(0.0, 0.4, 0.0))
    sd = scenes.cornell_box(seed=0)
    box = scenes.srt_matrix(translation=(0.3, 0.0, 0.6), scale=0.2, quat=scenes.euler_quaternion(0.1, 0.7, 0.0))
    with api.Builder() as b:
        mats = []
        for s in steps:
            payload = bytes.fromhex(s.get("hex", ""))
            if s["op"] == "resource":
                b.register_resource(payload)
            elif s["op"] == "call":
                b.register_call(s["symbol"], payload)
            elif s["op"] == "node":
                if s["traversal"] == 0x2000:
                    b.add_node_transform(s["traversal"], light_m)
                elif s["traversal"] == 0x3000:
                    b.add_node_transform(s["traversal"], cam_m)
                else:
                    b.add_node(s["traversal"], s["translation"])
            else:
                idx = b.add_program(s["kind"], s["symbol"], payload)
                if s["kind"] == 5:
                    mats.append(idx)
        m0 = sd.meshes[0]
        b.add_mesh(m0.vertices, m0.indices, mats[0])
        b.add_mesh(m0.vertices, m0.indices, mats[0], transform=box)
        sc, st = b.build(64, 64, 0, 4)
        exp = scenes.plane_transform(sd.planes[0], light_m)
        assert bytes(sc.planes[0]) == bytes(exp)
        assert list(sc.area_lights[0].translation) == [0.0, 0.0, 0.0]
        assert list(st.camera.position) == [float(x) for x in cam_m[[3, 7, 11]]]
        assert not sc.meshes[0].transform
        got = np.ctypeslib.as_array(C_float_ptr(sc.meshes[1].transform), (12,))
        assert np.array_equal(got, box)


def C_float_ptr(addr):
    import ctypes as C

    return C.cast(addr, C.POINTER(C.c_float))
