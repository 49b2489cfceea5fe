"""Writes scene descriptions in the reference renderer's JSON format (Src/PiperRenderer.cpp:150-362) for two of the
seeded scenes, so the scene-description path can be checked against the scenes built directly:

    python tests/golden/make_scene_json.py

tests/golden/scenes/cornell/   the Cornell box (scenes.cornell_box, seed 0): OBJ meshes, Matte surfaces with constant
                               textures, a Diffuse area light over a Plane, a zero environment, the camera as a sensor
                               node placed by its group transform
tests/golden/scenes/textured/  the textured room (scenes.textured_room, seed 0): checkerboard and image textures
                               (PPM / PGM), texture coordinates in the OBJ files
Each folder holds scene.json and options.json (the Render operator's options: ImageSize, SceneDesc, OutputDir).
Vertex values are written with the shortest decimal form of their float32 values, so they read back exactly.
"""
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from piper2_b200 import scenes  # noqa: E402

BC = "Piper.BuiltinComponent."
SURF = {1: "Matte", 2: "Plastic", 3: "Glass", 4: "Mirror", 5: "Substrate", 0: "BlackBody"}


def _f(x):
    return float(np.float32(x))


def write_obj(path, mesh):
    with open(path, "w") as fh:
        for v in mesh.vertices:
            fh.write("v " + " ".join(repr(_f(c)) for c in v) + "\n")
        if mesh.texcoords is not None:
            for t in mesh.texcoords:
                fh.write("vt " + " ".join(repr(_f(c)) for c in t) + "\n")
        for tri in mesh.indices:
            if mesh.texcoords is not None:
                fh.write("f " + " ".join(f"{i + 1}/{i + 1}" for i in tri) + "\n")
            else:
                fh.write("f " + " ".join(str(i + 1) for i in tri) + "\n")


def write_image(path, texels):
    t = np.asarray(texels, np.uint8)
    h, w, c = t.shape
    if c == 4:
        t, c = t[:, :, :3], 3
    with open(path, "wb") as fh:
        fh.write(f"{'P6' if c == 3 else 'P5'}\n{w} {h}\n255\n".encode())
        fh.write(t.tobytes())


def texture_desc(sd, folder, binding, const, channels, name):
    if binding:
        t = sd.textures[binding - 1]
        if t.kind == 1:
            return {"ClassID": BC + "ProceduralTexture.CheckBoard", "Scale": _f(t.scale),
                    "Black": [_f(x) for x in t.black[:t.channel]], "White": [_f(x) for x in t.white[:t.channel]]}
        ext = "ppm" if t.channel == 4 else "pgm"
        fname = f"{name}.{ext}"
        if t.channel == 4 and not np.all(t.texels[:, :, 3] == 255):
            raise ValueError("an RGBA image with alpha cannot be written as PPM")
        write_image(os.path.join(folder, fname), t.texels)
        return {"WrapMode": "Repeat" if t.wrap == 0 else "Mirror",
                "Image": {"ClassID": BC + "SampledTexture.Image", "Path": fname}}
    return {"ClassID": BC + "ProceduralTexture.ConstantTexture", "Value": [_f(x) for x in const[:channels]]}


def surface_desc(sd, folder, mat_index):
    m = sd.materials[mat_index]
    kind = SURF[m.type]
    c0, c1, r, tb = list(m.color0), list(m.color1), list(m.roughness), list(m.texture)
    slots = {"Matte": (("Diffuse", 0, 4), ("Roughness", 2, 1)),
             "Plastic": (("Diffuse", 0, 4), ("Specular", 1, 4), ("Roughness", 2, 1)),
             "Mirror": (("Reflection", 0, 4),),
             "Glass": (("Reflection", 0, 4), ("Transmission", 1, 4), ("RoughnessX", 2, 1), ("RoughnessY", 3, 1)),
             "Substrate": (("Diffuse", 0, 4), ("Specular", 1, 4), ("RoughnessX", 2, 1), ("RoughnessY", 3, 1)),
             "BlackBody": ()}[kind]
    d = {"ClassID": BC + "ClassicSurface." + kind}
    for key, slot, ch in slots:
        const = c0 if slot == 0 else c1 if slot == 1 else [r[slot - 2]]
        d[key] = texture_desc(sd, folder, tb[slot], const, ch, f"mat{mat_index}_{key}")
    return d


def scene_desc(sd, folder, sensor_mm, focal_mm):
    children = []
    for k, mesh in enumerate(sd.meshes):
        fname = f"mesh{k}.obj"
        write_obj(os.path.join(folder, fname), mesh)
        node = {"Type": "Instance", "Geometry": {"ClassID": BC + "TriangleMesh.TriangleMesh", "Path": fname},
                "Surface": surface_desc(sd, folder, mesh.material)}
        if any(mesh.translation):
            node["Transform"] = {"Translation": [_f(x) for x in mesh.translation]}
        children.append(node)
    children.append({"Type": "Instance", "ClassID": BC + "BasicLight.SampledEnvironment",
                     "Radiance": [_f(x) for x in sd.env_radiance]})
    for rad, first, count, tr in sd.area_lights:
        prims = [{"Origin": [_f(x) for x in p.origin], "U": [_f(x) for x in p.u], "V": [_f(x) for x in p.v]}
                 for p in sd.planes[first:first + count]]
        node = {"Type": "Instance", "ClassID": BC + "AreaLight.Diffuse", "Radiance": [_f(x) for x in rad],
                "Geometry": {"ClassID": BC + "BasicShapes.Plane", "Primitives": prims}}
        if any(tr):
            node["Transform"] = {"Translation": [_f(x) for x in tr]}
        children.append(node)
    st = sd.settings
    cam = st.camera
    children.append({"Type": "Group", "Transform": {"Translation": [_f(x) for x in cam.position]},
                     "Children": [{"Type": "Instance", "ID": "Camera", "ClassID": BC + "PerspectiveCamera.Sensor",
                                   "LookAt": [_f(x) for x in cam.look_at], "Up": [_f(x) for x in cam.up],
                                   "SensorSize": [sensor_mm, sensor_mm],
                                   "FocalLength": focal_mm,
                                   "FStop": 1e30}]})
    return {
        "Name": sd.name,
        "Objects": [],
        "Scene": {"Type": "Group", "Children": children},
        "LightSampler": {"ClassID": BC + "BasicLight.UniformLightSampler"},
        "Integrator": {"ClassID": BC + "PathTracing.Integrator", "MaxTraceDepth": int(st.max_depth),
                       "MinRussianRouletteDepth": int(st.min_rr_depth)},
        "Sampler": {"ClassID": BC + "ScrambledSobolSampler.Sampler", "SamplesPerPixel": int(st.samples_per_pixel),
                    "Scramble": False},
        "RenderDriver": {"ClassID": BC + "FixedSampler.Driver",
                         "Filter": {"ClassID": BC + "FixedSampler.SimpleFilter", "FilterType": "box"}},
        "Actions": [{"ActiveSensor": "Camera", "TimeBegin": 0.0, "ShutterOpenTime": 0.0, "ShutterCloseTime": 0.0,
                     "FrameCount": 1, "FitMode": "Fill"}],
    }


def main():
    # the camera of both scenes (scenes.cornell_box): 35 mm focal length, a square sensor for a 40 degree view
    focal_mm = 35.0
    sensor_mm = 2.0 * focal_mm * math.tan(math.radians(20.0))
    for name, sd in (("cornell", scenes.cornell_box(seed=0, width=32, height=32, spp=4)),
                     ("textured", scenes.textured_room(seed=0, width=32, height=32, spp=4))):
        folder = os.path.join(HERE, "scenes", name)
        os.makedirs(folder, exist_ok=True)
        with open(os.path.join(folder, "scene.json"), "w") as fh:
            json.dump(scene_desc(sd, folder, sensor_mm, focal_mm), fh, indent=1)
        with open(os.path.join(folder, "options.json"), "w") as fh:
            json.dump({"ImageSize": [sd.settings.width, sd.settings.height], "SceneDesc": "scene.json",
                       "SceneParser": "Piper.Infrastructure.JSONSerializer.JSONSerializer",
                       "Tracer": {"ClassID": "Piper.B200.Tracer"}, "OutputDir": "out"}, fh, indent=1)
        print(folder)


if __name__ == "__main__":
    main()
