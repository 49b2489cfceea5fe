"""Generates tests/golden/payloads.json: the materialized component programs of two scenes, with every payload
written by the reference's own POD types (tests/golden/payloads_ref.cpp compiled against a Piper2 checkout).

    python tests/golden/make_payloads.py /path/to/Piper2      (or PIPER2_REFERENCE=/path/to/Piper2)

Each scene is a list of steps in the order a Piper tracer would see them while its components materialize
(Tracer.hpp:86-91, 121-133):
    {"op": "resource", "hex": ...}                          MaterializeContext::registerResource
    {"op": "call", "symbol": ..., "hex": ..., "handle": h}    MaterializeContext::registerCall (h: the handle
                                                             the builder must return, 1, 2, ... in order)
    {"op": "node", "traversal": t, "translation": [x, y, z]} Tracer::buildNode
    {"op": "program", "kind": k, "symbol": ..., "hex": ...} a component's program and payload
The meshes are not payloads (geometry buffers): the test takes them from the same scene generator.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from piper2_b200 import capi, scenes  # noqa: E402

KIND = {"sensor": 0, "integrator": 1, "driver": 2, "sampler": 3, "light_sampler": 4, "surface": 5, "light": 6}
SURFACE_INIT = {1: "matteInit", 2: "plasticInit", 3: "glassInit", 4: "mirrorInit", 5: "substrateInit",
                0: "blackBodyInit"}


def _f(v):
    return " ".join(repr(float(x)) for x in v)


class Steps:
    def __init__(self, tool):
        self.tool = tool
        self.steps = []
        self.calls = 0
        self.resources = 0

    def payload(self, request):
        out = subprocess.run([self.tool], input=request + "\n", capture_output=True, text=True, check=True).stdout
        size, hx = out.split()
        assert int(size) * 2 == len(hx)
        return hx

    def resource(self, data: bytes):
        self.steps.append({"op": "resource", "hex": data.hex()})
        self.resources += 1
        return self.resources - 1

    def call(self, symbol, request):
        self.calls += 1
        self.steps.append({"op": "call", "symbol": symbol, "hex": self.payload(request) if request else "",
                           "handle": self.calls})
        return self.calls

    def node(self, traversal, translation):
        self.steps.append({"op": "node", "traversal": traversal, "translation": [float(x) for x in translation]})

    def program(self, kind, symbol, request=None):
        self.steps.append({"op": "program", "kind": KIND[kind], "symbol": symbol,
                           "hex": self.payload(request) if request else ""})


def scene_steps(tool, sd, filt="box", alpha=2.0):
    s = Steps(tool)
    # lights[0] is the environment (Embree.cpp:1174-1188), then the area lights in order
    s.node(0x1000, (0, 0, 0))
    s.program("light", "SEInit", f"environment {0x1000} {_f(sd.env_radiance)}")
    for li, (rad, first, count, trans) in enumerate(sd.area_lights):
        planes = sd.planes[first:first + count]
        blob = b"".join(bytes.fromhex(s.payload(f"plane {_f(p.origin)} {_f(p.u)} {_f(p.v)} {_f(p.normal)} "
                                                 f"{_f(p.tangent)} {p.max_det_comp}")) for p in planes)
        prim = s.resource(blob)
        cdf = s.resource(np.zeros(count, np.float32).tobytes())
        pdf = s.resource(np.zeros(count, np.float32).tobytes())
        trav = 0x2000 + li
        s.node(trav, trans)
        h = s.call("planeSample", f"cdf {prim} {trav} {cdf} {pdf} 1.0 {count}")
        s.program("light", "diffuseInit", f"diffuse {_f(rad)} {h} 1.0")
    for m in sd.materials:
        c0 = s.call("constantTexture", f"constant 4 {_f(m.color0)}")
        c1 = s.call("constantTexture", f"constant 4 {_f(m.color1)}")
        r0 = s.call("constantTexture", f"constant 1 {m.roughness[0]!r} 0 0 0")
        r1 = s.call("constantTexture", f"constant 1 {m.roughness[1]!r} 0 0 0")
        req = {1: f"matte {c0} {r0}", 2: f"plastic {c0} {c1} {r0}", 3: f"glass {c0} {c1} {r0} {r1}",
               4: f"mirror {c0}", 5: f"substrate {c0} {c1} {r0} {r1}", 0: None}[m.type]
        s.program("surface", SURFACE_INIT[m.type], req)
    cam = sd.settings.camera
    s.node(0x3000, cam.position)
    s.program("sensor", "rayGen", f"camera {0x3000} {_f(cam.look_at)} {_f(cam.sensor_size)} {_f(cam.up)} "
                                  f"{cam.focal_length!r} {cam.aperture_radius!r}")
    st = sd.settings
    s.program("integrator", "trace", f"pathtracing {st.max_depth} {st.min_rr_depth} 11 12 13")
    fh = s.call(filt, f"gaussian {-alpha!r} {float(np.exp(-alpha))!r}")
    s.program("driver", "accumulate", f"driver {fh}")
    s.program("sampler", "sobolStart")
    s.program("light_sampler", "uniformSelect")
    return s.steps


def six_materials():
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


SCENES = {
    "cornell_box": (lambda: scenes.cornell_box(seed=0), "box"),
    "six_materials_gaussian": (six_materials, "gaussian"),
}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PIPER2_REFERENCE")
    if not ref or not os.path.isdir(os.path.join(ref, "Src", "BuiltinComponent")):
        raise SystemExit("pass the Piper2 checkout or set PIPER2_REFERENCE")
    with tempfile.TemporaryDirectory() as tmp:
        tool = os.path.join(tmp, "payloads_ref")
        subprocess.run(["g++", "-std=c++17", "-w", "-include", "cstddef", "-include", "cstring", "-include", "algorithm",
                        "-include", "cmath", "-I", os.path.join(ref, "Src"), "-o", tool,
                        os.path.join(HERE, "payloads_ref.cpp")], check=True)
        out = {}
        for name, (make, filt) in SCENES.items():
            sd = make()
            out[name] = scene_steps(tool, sd, filt, float(sd.settings.gaussian_alpha))
    with open(os.path.join(HERE, "payloads.json"), "w") as f:
        json.dump(out, f, indent=0)
    print("payload fixture written")


if __name__ == "__main__":
    main()
