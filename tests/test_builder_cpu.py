"""The drop-in boundary on the Piper side: component programs as a Piper tracer receives them (symbol names and
payload bytes written by the reference's own POD types; tests/golden/payloads.json, made by
tests/golden/make_payloads.py) become, through the library's pb2_builder_*, exactly the scene and render settings
that the scene generator describes directly.  Host-side only: runs without a GPU."""
import json
import os

import numpy as np
import pytest

from piper2_b200 import capi, scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "payloads.json")


def _api():
    from piper2_b200 import api

    return api


def _six_materials():
    sd = scenes.cornell_box(seed=6, width=24, height=24, spp=8)
    sd.materials = [scenes.material("Plastic", (0.4, 0.4, 0.4), (0.5, 0.5, 0.5), (0.3, 0)),
                    scenes.material("Matte", (0.65, 0.05, 0.05), roughness=(0.4, 0)),
                    scenes.material("Substrate", (0.12, 0.45, 0.15), (0.2, 0.2, 0.2), (0.2, 0.3)),
                    scenes.material("Glass", (1, 1, 1), (1, 1, 1), (0, 0)),
                    scenes.material("Glass", (1, 1, 1), (1, 1, 1), (0.2, 0.2)),
                    scenes.material("Mirror", (0.9, 0.9, 0.9))]
    sd.meshes[5].material = 3
    sd.meshes[6].material = 4
    sd.meshes[2].material = 5
    sd.settings.filter = capi.FILTER["gaussian"]
    sd.settings.gaussian_alpha = 2.0
    return sd


SCENES = {"cornell_box": lambda: scenes.cornell_box(seed=0), "six_materials_gaussian": _six_materials}


def replay(name, sd=None):
    """A Builder fed the fixture's steps for scene `name`, plus the scene's meshes, built at its settings."""
    with open(GOLDEN) as f:
        steps = json.load(f)[name]
    sd = sd or SCENES[name]()
    b = _api().Builder()
    materials = []
    for s in steps:
        payload = bytes.fromhex(s.get("hex", ""))
        if s["op"] == "resource":
            b.register_resource(payload)
        elif s["op"] == "call":
            assert b.register_call(s["symbol"], payload) == s["handle"]
        elif s["op"] == "node":
            b.add_node(s["traversal"], s["translation"])
        else:
            idx = b.add_program(s["kind"], s["symbol"], payload)
            if s["kind"] == 5:
                materials.append(idx)
    for m in sd.meshes:
        b.add_mesh(m.vertices, m.indices, materials[m.material], m.translation)
    st = sd.settings
    b.build(st.width, st.height, st.fit_mode, st.samples_per_pixel)
    return b, sd


def _bytes(x):
    return bytes(x)


@pytest.mark.parametrize("name", sorted(SCENES))
def test_payloads_build_the_generators_scene(name):
    b, sd = replay(name)
    sc, st = b.scene, b.settings
    ref_sc, keep = sd.to_ctypes()
    if st.filter != capi.FILTER["gaussian"]:  # the box and triangle filters have no parameter
        st.gaussian_alpha = sd.settings.gaussian_alpha
    assert _bytes(st) == _bytes(sd.settings)  # camera, filter, depths, film: byte for byte
    assert sc.material_count == len(sd.materials)
    for i in range(sc.material_count):
        assert _bytes(sc.materials[i]) == _bytes(sd.materials[i]), i
    assert sc.plane_count == len(sd.planes)
    for i in range(sc.plane_count):
        assert _bytes(sc.planes[i]) == _bytes(sd.planes[i]), i
    assert sc.area_light_count == ref_sc.area_light_count
    for i in range(sc.area_light_count):
        assert _bytes(sc.area_lights[i]) == _bytes(ref_sc.area_lights[i]), i
    assert list(sc.env_radiance) == list(ref_sc.env_radiance)
    assert sc.mesh_count == ref_sc.mesh_count
    for i in range(sc.mesh_count):
        a, r = sc.meshes[i], ref_sc.meshes[i]
        assert (a.vert_count, a.tri_count, a.material) == (r.vert_count, r.tri_count, r.material)
        va = np.ctypeslib.as_array(C_float_ptr(a.vertices), (a.vert_count * 3,))
        assert np.array_equal(va, np.asarray(sd.meshes[i].vertices, np.float32).reshape(-1))
        ia = np.ctypeslib.as_array(C_u32_ptr(a.indices), (a.tri_count * 3,))
        assert np.array_equal(ia, np.asarray(sd.meshes[i].indices, np.uint32).reshape(-1))
    b.close()


def C_float_ptr(addr):
    import ctypes as C

    return C.cast(addr, C.POINTER(C.c_float))


def C_u32_ptr(addr):
    import ctypes as C

    return C.cast(addr, C.POINTER(C.c_uint32))


def test_unknown_symbols_are_rejected():
    """As the reference's pipeline build fails on a program it cannot link: the symbol is named."""
    api = _api()
    with api.Builder() as b:
        for kind, sym in (("surface", "disneyPrincipledBRDFInit"), ("light", "pointInit"), ("sensor", "orthoRayGen"),
                          ("integrator", "ambientOcclusion"), ("driver", "adaptiveAccumulate")):
            with pytest.raises(capi.PB2Error, match=sym):
                b.add_program(kind, sym, b"\0" * 32)
        h = b.register_call("sampleTexture", b"\0" * 16)
        with pytest.raises(capi.PB2Error, match="sampleTexture"):
            b.add_program("surface", "matteInit", h.to_bytes(8, "little") + h.to_bytes(8, "little"))
        f = b.register_call("mitchell", b"")
        with pytest.raises(capi.PB2Error, match="mitchell"):
            b.add_program("driver", "accumulate", f.to_bytes(8, "little"))


def test_payload_size_and_order_are_checked():
    api = _api()
    with api.Builder() as b:
        with pytest.raises(capi.PB2Error, match="48"):
            b.add_program("sensor", "rayGen", b"\0" * 40)  # PCData is 48 bytes
        with pytest.raises(capi.PB2Error, match="environment"):  # lights[0] must be the environment
            b.add_program("light", "diffuseInit", b"\0" * 32)
        with pytest.raises(capi.PB2Error, match="no a sensor|has no"):
            b.build(16, 16, 0, 4)
