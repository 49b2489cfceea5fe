"""Scene description -> pipeline -> frames: the reference's Render operator (Src/PiperRenderer.cpp:150-362) for the
render path this library implements.

A scene description is the JSON document the reference's renderer reads (its ConfigSerializer,
PiperRenderer.cpp:291-296): components are objects with a "ClassID" of the form "<module>.<class>" (the module
names of Src/Module.json, split at the last dot as the module loader does, PiperCore.cpp:386-397) and their
constructors' keys; the scene itself is a tree of "Group" and "Instance" nodes (PiperRenderer.cpp:150-211):

    {"Objects": [...],                                   # instantiated up front, by "ID" (:252-255)
     "Scene": {"Type": "Group", "Children": [
         {"Type": "Instance", "Geometry": {...}, "Surface": {...}, "Transform": {...}},     # a GSM instance
         {"Type": "Instance", "ClassID": "Piper.BuiltinComponent.AreaLight.Diffuse", ...},   # a light
         {"Type": "Instance", "ClassID": "Piper.BuiltinComponent.PerspectiveCamera.Sensor", "ID": "Camera", ...}]},
     "LightSampler": {...}, "Integrator": {...}, "Sampler": {...}, "RenderDriver": {...},
     "Actions": [{"ActiveSensor": "Camera", "TimeBegin": 0, "ShutterOpenTime": 0, "ShutterCloseTime": 0,
                  "FrameCount": 1, "FitMode": "Fill"}]}

A group child's "Transform" holds "Translation", "Scale" (a number, three numbers, or {"Scale", "Skew", "Shift"})
and "Rotation" (three Euler angles or a quaternion w, x, y, z) (PiperRenderer.cpp:58-141).

Components understood (their keys as the reference's constructors read them):

* Geometry: ``Piper.BuiltinComponent.TriangleMesh.TriangleMesh`` {"Path"} -- the reference imports any format
  through assimp (TriangleMesh.cpp:40-123), which is not available here: Wavefront OBJ (v, vt, f; polygons
  fanned into triangles, identical (position, texcoord) pairs joined) and .npz (``vertices``, ``indices``,
  optional ``texcoords``) are read; ``Piper.BuiltinComponent.BasicShapes.Plane`` {"Primitives": [{"Origin",
  "U", "V"}]} as the geometry of area lights.
* Surface: ``Piper.BuiltinComponent.ClassicSurface.{BlackBody, Matte, Plastic, Mirror, Glass, Substrate}`` with
  textures "Diffuse", "Roughness", "Specular", "Reflection", "Transmission", "RoughnessX", "RoughnessY"
  (Classic.cpp:70-199); a texture is ``...ProceduralTexture.ConstantTexture`` {"Value"},
  ``...ProceduralTexture.CheckBoard`` {"Scale", "Black", "White"}, or a sampled image {"WrapMode", "Image":
  {"ClassID": "...SampledTexture.Image", "Path"}} (Embree.cpp:1335-1351; images read from binary PPM / PGM or
  .npy of uint8).
* Light: ``Piper.BuiltinComponent.AreaLight.Diffuse`` {"Radiance", "Geometry"}, ``Piper.BuiltinComponent.
  BasicLight.SampledEnvironment`` {"Radiance"} (exactly one, the reference's lights[0], Embree.cpp:1174-1188).
* Sensor: ``Piper.BuiltinComponent.PerspectiveCamera.Sensor`` {"LookAt", "SensorSize", "Up", "FocalLength",
  "FStop"}, placed at its node's origin (PerspectiveCamera/Kernel.cpp:25-28).
* ``...BasicLight.UniformLightSampler``, ``...PathTracing.Integrator`` {"MaxTraceDepth",
  "MinRussianRouletteDepth"}, ``...ScrambledSobolSampler.Sampler`` {"SamplesPerPixel", "Scramble"},
  ``...FixedSampler.Driver`` {"Filter": {"ClassID": "...FixedSampler.SimpleFilter", "FilterType", "Alpha"}}.

Anything else fails naming it, as the reference's loader and pipeline build fail on a class they cannot resolve
or link.  Dynamic (keyframed) transforms are rejected: motion is not rendered.  ``Scramble: true`` selects the
library's Owen-scrambled Sobol extension (the reference aborts on it, ScrambledSobolSampler.cpp:51-53).

Frames are written as PFM (the reference writes OpenEXR, PiperRenderer.cpp:269-302, which is not available
here) to ``<OutputDir>/Action<k>/Frame<i>.pfm``; pixels that are not finite or are negative become (1, 0, 0)
with a warning, as the reference's writer does.
"""
from __future__ import annotations

import json
import math
import os
import warnings
from dataclasses import dataclass, field

import numpy as np

from . import capi, scenes

f32 = np.float32
BC = "Piper.BuiltinComponent."


class SceneError(ValueError):
    """An invalid or unsupported scene description (the reference raises through its error handler)."""


def _split_class(cfg) -> tuple:
    cid = cfg.get("ClassID") if isinstance(cfg, dict) else None
    if not isinstance(cid, str) or "." not in cid:
        raise SceneError(f"Invalid classID \"{cid}\".")
    pos = cid.rfind(".")
    return cid[:pos], cid[pos + 1:]


def _vec(v, n=3, what="vector"):
    if not isinstance(v, (list, tuple)) or len(v) != n:
        raise SceneError(f"{what} must hold {n} numbers")
    return [float(x) for x in v]


@dataclass
class Transform:
    """A node transform: translation-only (matrix None) or a general 3x4 local-to-world matrix."""
    translation: tuple = (0.0, 0.0, 0.0)
    matrix: np.ndarray | None = None  # (3, 4) float64

    def compose(self, child: "Transform") -> "Transform":
        if self.matrix is None and child.matrix is None:
            t = tuple(float(f32(a) + f32(b)) for a, b in zip(self.translation, child.translation))
            return Transform(t)
        a, b = self.as_matrix(), child.as_matrix()
        m = np.zeros((3, 4))
        m[:, :3] = a[:, :3] @ b[:, :3]
        m[:, 3] = a[:, :3] @ b[:, 3] + a[:, 3]
        return Transform(tuple(m[:, 3]), m)

    def as_matrix(self) -> np.ndarray:
        if self.matrix is not None:
            return self.matrix
        m = np.zeros((3, 4))
        m[:, :3] = np.eye(3)
        m[:, 3] = self.translation
        return m

    def origin(self):
        return tuple(float(x) for x in self.translation)


def parse_transform(cfg) -> Transform:
    """PiperRenderer.cpp:58-141: Translation, Scale (number | [3] | {Scale, Skew, Shift}), Rotation (Euler angles
    pitch, yaw, roll | quaternion w, x, y, z)."""
    if not isinstance(cfg, dict):
        raise SceneError("Invalid transform")
    if "Offset" in cfg:
        raise SceneError("dynamic (keyframed) transforms are not supported: motion is not rendered")
    tr = _vec(cfg.get("Translation", [0, 0, 0]), 3, "Translation")
    scale, skew, shift = [1.0, 1.0, 1.0], [0.0, 0.0, 0.0], [0.0, 0.0, 0.0]
    if "Scale" in cfg:
        s = cfg["Scale"]
        if isinstance(s, (int, float)):
            scale = [float(s)] * 3
        elif isinstance(s, list):
            scale = _vec(s, 3, "Scale")
        elif isinstance(s, dict):
            scale = _vec(s["Scale"], 3, "Scale")
            skew = _vec(s["Skew"], 3, "Skew")
            shift = _vec(s["Shift"], 3, "Shift")
        else:
            raise SceneError("Invalid transform")
    quat = (1.0, 0.0, 0.0, 0.0)
    if "Rotation" in cfg:
        r = cfg["Rotation"]
        if isinstance(r, list) and len(r) == 3:
            quat = scenes.euler_quaternion(*[float(x) for x in r])
        elif isinstance(r, list) and len(r) == 4:
            quat = tuple(float(x) for x in r)
        else:
            raise SceneError("Invalid transform")
    if scale == [1.0, 1.0, 1.0] and skew == [0.0] * 3 and shift == [0.0] * 3 and tuple(quat) == (1.0, 0.0, 0.0, 0.0):
        return Transform(tuple(tr))
    m = np.asarray(scenes.srt_matrix(scenes.srt(tuple(tr), tuple(scale), tuple(quat), tuple(skew), tuple(shift))),
                   dtype=np.float64).reshape(3, 4)
    return Transform(tuple(tr), m)


# ---- assets -----------------------------------------------------------------------------------------------------

def load_obj(path: str):
    """Wavefront OBJ -> (vertices (V, 3) float32, indices (T, 3) uint32, texcoords (V, 2) float32 or None): one
    mesh (the reference accepts only one, TriangleMesh.cpp:57-58), polygons fanned into triangles, identical
    (position, texcoord) corners joined (assimp's Triangulate | JoinIdenticalVertices)."""
    pos, uv, corners, faces = [], [], {}, []
    out_v, out_t = [], []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if not parts or parts[0].startswith("#"):
                continue
            if parts[0] == "v":
                pos.append([float(x) for x in parts[1:4]])
            elif parts[0] == "vt":
                uv.append([float(x) for x in parts[1:3]])
            elif parts[0] == "f":
                ids = []
                for c in parts[1:]:
                    fields = c.split("/")
                    vi = int(fields[0])
                    vi = vi - 1 if vi > 0 else len(pos) + vi
                    ti = None
                    if len(fields) > 1 and fields[1]:
                        ti = int(fields[1])
                        ti = ti - 1 if ti > 0 else len(uv) + ti
                    key = (vi, ti)
                    if key not in corners:
                        if not 0 <= vi < len(pos) or (ti is not None and not 0 <= ti < len(uv)):
                            raise SceneError(f"{path}: face index out of range")
                        corners[key] = len(out_v)
                        out_v.append(pos[vi])
                        out_t.append(uv[ti] if ti is not None else None)
                    ids.append(corners[key])
                if len(ids) < 3:
                    raise SceneError(f"{path}: a face with fewer than three corners")
                for k in range(1, len(ids) - 1):
                    faces.append([ids[0], ids[k], ids[k + 1]])
    if not faces:
        raise SceneError(f"Failed to load scene {path} : no faces")
    v = np.asarray(out_v, dtype=np.float32).reshape(-1, 3)
    ix = np.asarray(faces, dtype=np.uint32).reshape(-1, 3)
    tc = None
    if any(t is not None for t in out_t):
        if any(t is None for t in out_t):
            raise SceneError(f"{path}: texture coordinates on some corners only")
        tc = np.asarray(out_t, dtype=np.float32).reshape(-1, 2)
    return v, ix, tc


def load_mesh(path: str):
    ext = os.path.splitext(path)[1].lower()
    if ext == ".obj":
        return load_obj(path)
    if ext == ".npz":
        z = np.load(path)
        tc = np.asarray(z["texcoords"], np.float32).reshape(-1, 2) if "texcoords" in z.files else None
        return (np.asarray(z["vertices"], np.float32).reshape(-1, 3), np.asarray(z["indices"], np.uint32).reshape(-1, 3),
                tc)
    raise SceneError(f"Failed to load scene {path} : only Wavefront OBJ and .npz meshes are read (no assimp)")


def load_image(path: str) -> np.ndarray:
    """An 8-bit image (H, W, C) from binary PPM (P6) / PGM (P5) or a .npy of uint8."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".npy":
        a = np.load(path)
        if a.dtype != np.uint8:
            raise SceneError(f"{path}: an image array must be uint8")
        return a
    with open(path, "rb") as fh:
        data = fh.read()
    tokens, pos = [], 0
    while len(tokens) < 4:
        while data[pos:pos + 1].isspace():
            pos += 1
        if data[pos:pos + 1] == b"#":
            pos = data.index(b"\n", pos) + 1
            continue
        end = pos
        while not data[end:end + 1].isspace():
            end += 1
        tokens.append(data[pos:end])
        pos = end
    pos += 1
    magic, w, h, mx = tokens[0], int(tokens[1]), int(tokens[2]), int(tokens[3])
    if magic not in (b"P5", b"P6") or mx != 255:
        raise SceneError(f"{path}: only binary 8-bit PPM (P6) and PGM (P5) images are read")
    c = 3 if magic == b"P6" else 1
    return np.frombuffer(data, np.uint8, w * h * c, pos).reshape(h, w, c).copy()


# ---- the scene ----------------------------------------------------------------------------------------------------

@dataclass
class Sensor:
    config: dict
    transform: Transform


@dataclass
class Action:
    active_sensor: str
    time_begin: float
    shutter_open: float
    shutter_close: float
    frame_count: int
    fit_mode: str


@dataclass
class LoadedScene:
    scene: scenes.SceneData
    sensors: dict = field(default_factory=dict)   # ID -> Sensor
    actions: list = field(default_factory=list)
    spp: int = 1
    scramble: int = 0
    max_depth: int = 1
    min_rr_depth: int = 0
    filter: str = "box"
    alpha: float = 2.0

    def settings(self, sensor_id: str, width: int, height: int, fit_mode: str = "Fill") -> capi.RenderSettings:
        """Pipeline::prepare(sensor, width, height, fitMode): the render settings of one view."""
        s = self.sensors.get(sensor_id)
        if s is None:
            raise SceneError(f"Failed to find a node with sensor named \"{sensor_id}\".")
        c = s.config
        try:
            cam = scenes.camera_from_config(s.transform.origin(), _vec(c["LookAt"], 3, "LookAt"), _vec(c["Up"], 3, "Up"),
                                            _vec(c["SensorSize"], 2, "SensorSize"), float(c["FocalLength"]),
                                            float(c["FStop"]))
        except KeyError as e:
            raise SceneError(f"sensor \"{sensor_id}\" lacks {e.args[0]}") from None
        if fit_mode not in capi.FIT:
            raise SceneError(f"Invalid FitMode \"{fit_mode}\".")
        return scenes.render_settings(width, height, self.spp, self.max_depth, self.min_rr_depth, cam, self.filter,
                                      self.alpha, fit_mode, self.scramble)

    def scene_for(self, sensor_id: str, width: int, height: int, fit_mode: str = "Fill") -> scenes.SceneData:
        sd = scenes.SceneData(meshes=self.scene.meshes, planes=self.scene.planes, area_lights=self.scene.area_lights,
                              materials=self.scene.materials, textures=self.scene.textures,
                              env_radiance=self.scene.env_radiance, name=self.scene.name)
        sd.settings = self.settings(sensor_id, width, height, fit_mode)
        return sd


_TEXTURE_SLOTS = {
    # surface class -> (config key, material slot: 0 color0, 1 color1, 2 roughness[0], 3 roughness[1], channels)
    "BlackBody": (),
    "Matte": (("Diffuse", 0, 4), ("Roughness", 2, 1)),
    "Plastic": (("Diffuse", 0, 4), ("Specular", 1, 4), ("Roughness", 2, 1)),
    "Mirror": (("Reflection", 0, 4),),
    "Glass": (("Reflection", 0, 4), ("Transmission", 1, 4), ("RoughnessX", 2, 1), ("RoughnessY", 3, 1)),
    "Substrate": (("Diffuse", 0, 4), ("Specular", 1, 4), ("RoughnessX", 2, 1), ("RoughnessY", 3, 1)),
}


class _Loader:
    def __init__(self, base_dir: str):
        self.base = base_dir
        self.sd = scenes.SceneData()
        self.sensors = {}
        self.env = None
        self.meshes = {}

    def path(self, p):
        return p if os.path.isabs(p) else os.path.join(self.base, p)

    # textures (Tracer::generateTexture, Embree.cpp:1335-1351, 1424-1430)
    def texture(self, cfg, channel: int, what: str):
        if not isinstance(cfg, dict):
            raise SceneError(f"{what}: a texture description is an object")
        if "ClassID" in cfg:
            mod, cls = _split_class(cfg)
            if mod == BC + "ProceduralTexture" and cls == "ConstantTexture":
                val = [float(x) for x in cfg["Value"]]
                if len(val) not in (1, 2, 4):
                    raise SceneError(f"Unsupported channel {len(val)}")
                if len(val) != channel:
                    raise SceneError(f"Mismatched channel. Expect {channel}, but get {len(val)} ({what})")
                return ("const", val)
            if mod == BC + "ProceduralTexture" and cls == "CheckBoard":
                black, white = [float(x) for x in cfg["Black"]], [float(x) for x in cfg["White"]]
                if len(black) != channel:
                    raise SceneError(f"Mismatched channel. Expect {channel}, but get {len(black)} ({what})")
                return ("tex", scenes.checkerboard(float(cfg["Scale"]), black, white))
            raise SceneError(f"unsupported texture class \"{cfg['ClassID']}\" ({what})")
        wrap = cfg.get("WrapMode")
        if wrap not in capi.WRAP:
            raise SceneError(f"Unrecognized wrap mode {wrap}")
        img = cfg.get("Image")
        if not isinstance(img, dict) or _split_class(img) != (BC + "SampledTexture", "Image"):
            raise SceneError(f"{what}: a sampled texture's \"Image\" is a {BC}SampledTexture.Image")
        t = scenes.image_texture(load_image(self.path(img["Path"])), wrap)
        if t.channel != channel:
            raise SceneError(f"Mismatched channel. Expect {channel}, but get {t.channel} ({what})")
        return ("tex", t)

    def surface(self, cfg) -> int:
        mod, cls = _split_class(cfg)
        if mod != BC + "ClassicSurface" or cls not in _TEXTURE_SLOTS:
            raise SceneError(f"unsupported surface class \"{cfg['ClassID']}\"")
        colors = [[0.0] * 4, [0.0] * 4]
        rough = [0.0, 0.0]
        binding = [0, 0, 0, 0]
        for key, slot, ch in _TEXTURE_SLOTS[cls]:
            if key not in cfg:
                raise SceneError(f"surface {cls} lacks \"{key}\"")
            kind, val = self.texture(cfg[key], ch, f"{cls}.{key}")
            if kind == "tex":
                self.sd.textures.append(val)
                binding[slot] = len(self.sd.textures)
            elif slot < 2:
                colors[slot] = val
            else:
                rough[slot - 2] = val[0]
        self.sd.materials.append(scenes.material(cls, colors[0], colors[1], tuple(rough), tuple(binding)))
        return len(self.sd.materials) - 1

    def planes(self, geom, tf: Transform, what: str):
        mod, cls = _split_class(geom)
        if (mod, cls) != (BC + "BasicShapes", "Plane"):
            raise SceneError(f"{what}: only {BC}BasicShapes.Plane geometry is supported for area lights")
        out = []
        for p in geom["Primitives"]:
            pl = scenes.plane_make(_vec(p["Origin"], 3, "Origin"), _vec(p["U"], 3, "U"), _vec(p["V"], 3, "V"))
            if tf.matrix is not None:
                pl = scenes.plane_transform(pl, np.asarray(tf.matrix, np.float32).reshape(12))
            out.append(pl)
        if not out:
            raise SceneError(f"{what}: a Plane geometry without primitives")
        return out

    def instance(self, cfg, tf: Transform):
        if "ClassID" in cfg:
            mod, cls = _split_class(cfg)
            if (mod, cls) == (BC + "PerspectiveCamera", "Sensor"):
                return ("sensor", cfg)
            if (mod, cls) == (BC + "AreaLight", "Diffuse"):
                planes = self.planes(cfg["Geometry"], tf, "Diffuse area light")
                first = len(self.sd.planes)
                self.sd.planes += planes
                trans = tf.translation if tf.matrix is None else (0.0, 0.0, 0.0)
                self.sd.area_lights.append((tuple(_vec(cfg["Radiance"], 3, "Radiance")), first, len(planes), trans))
                return ("light", None)
            if (mod, cls) == (BC + "BasicLight", "SampledEnvironment"):
                if self.env is not None:
                    raise SceneError("only one environment light is supported (it is the reference's lights[0])")
                self.env = tuple(_vec(cfg["Radiance"], 3, "Radiance"))
                return ("light", None)
            raise SceneError(f"unsupported scene object \"{cfg['ClassID']}\"")
        geom, surf = cfg.get("Geometry"), cfg.get("Surface")
        if geom is None or surf is None:
            raise SceneError("Invalid scene node.")
        mod, cls = _split_class(geom)
        if (mod, cls) != (BC + "TriangleMesh", "TriangleMesh"):
            raise SceneError(f"unsupported geometry class \"{geom['ClassID']}\" for a surface instance")
        key = self.path(geom["Path"])
        if key not in self.meshes:
            self.meshes[key] = load_mesh(key)
        v, ix, tc = self.meshes[key]
        mat = self.surface(surf)
        self.sd.meshes.append(scenes.MeshData(v, ix, mat, translation=tf.translation if tf.matrix is None else
                                              (0.0, 0.0, 0.0),
                                              transform=None if tf.matrix is None else
                                              np.asarray(tf.matrix, np.float32).reshape(12), texcoords=tc))
        return ("mesh", None)

    # Render::buildScene (PiperRenderer.cpp:150-211)
    def node(self, cfg, tf: Transform):
        if not isinstance(cfg, dict) or "Type" not in cfg:
            raise SceneError("Invalid scene node.")
        kind = cfg["Type"]
        if kind == "Instance":
            res = self.instance(cfg, tf)
            if "ID" in cfg and res[0] == "sensor":
                self.sensors[cfg["ID"]] = Sensor(res[1], tf)
            return
        if kind == "Group":
            for child in cfg.get("Children", []):
                ctf = parse_transform(child["Transform"]) if isinstance(child, dict) and "Transform" in child \
                    else Transform()
                self.node(child, tf.compose(ctf))
            return
        raise SceneError("Invalid scene node.")


def _component(cfg, module: str, cls: str, what: str):
    if not isinstance(cfg, dict):
        raise SceneError(f"{what}: a component description is an object")
    got = _split_class(cfg)
    if got != (BC + module, cls):
        raise SceneError(f"{what}: unsupported class \"{cfg['ClassID']}\" (expected {BC}{module}.{cls})")
    return cfg


def load(desc, base_dir: str | None = None) -> LoadedScene:
    """Parses a scene description (a dict, or the path of a JSON file) into a :class:`LoadedScene`."""
    if isinstance(desc, (str, os.PathLike)):
        base_dir = base_dir or os.path.dirname(os.path.abspath(desc))
        with open(desc) as fh:
            desc = json.load(fh)
    if not isinstance(desc, dict):
        raise SceneError("a scene description is a JSON object")
    ld = _Loader(base_dir or os.getcwd())
    # Objects: instantiated up front by ID (PiperRenderer.cpp:252-255); their classes must resolve
    ids = set()
    for obj in desc.get("Objects", []):
        _split_class(obj)
        if "ID" not in obj:
            raise SceneError("an entry of Objects has no ID")
        ids.add(obj["ID"])
    for key in ("Scene", "LightSampler", "Integrator", "Sampler", "RenderDriver", "Actions"):
        if key not in desc:
            raise SceneError(f"the scene description lacks \"{key}\"")
    ld.node(desc["Scene"], Transform())
    if ld.env is None:
        # the pipeline needs the environment as lights[0] (Embree.cpp:1174-1188)
        raise SceneError(f"the scene needs one {BC}BasicLight.SampledEnvironment light")
    ld.sd.env_radiance = ld.env
    _component(desc["LightSampler"], "BasicLight", "UniformLightSampler", "LightSampler")
    integ = _component(desc["Integrator"], "PathTracing", "Integrator", "Integrator")
    samp = _component(desc["Sampler"], "ScrambledSobolSampler", "Sampler", "Sampler")
    drv = _component(desc["RenderDriver"], "FixedSampler", "Driver", "RenderDriver")
    filt = _component(drv.get("Filter"), "FixedSampler", "SimpleFilter", "RenderDriver.Filter")
    ftype = filt.get("FilterType")
    if ftype not in capi.FILTER:
        raise SceneError(f"unsupported FilterType \"{ftype}\" (box, triangle or gaussian)")
    out = LoadedScene(ld.sd, ld.sensors)
    out.max_depth = int(integ["MaxTraceDepth"])
    out.min_rr_depth = int(integ["MinRussianRouletteDepth"])
    out.spp = int(samp["SamplesPerPixel"])
    out.scramble = 1 if samp.get("Scramble", False) else 0
    out.filter = ftype
    out.alpha = float(filt.get("Alpha", 2.0))
    # Actions (PiperRenderer.cpp:235-247)
    for a in desc["Actions"]:
        try:
            out.actions.append(Action(str(a["ActiveSensor"]), float(a["TimeBegin"]), float(a["ShutterOpenTime"]),
                                      float(a["ShutterCloseTime"]), int(a["FrameCount"]), str(a["FitMode"])))
        except KeyError as e:
            raise SceneError(f"an action lacks {e.args[0]}") from None
        if out.actions[-1].fit_mode not in capi.FIT:
            raise SceneError(f"Invalid FitMode \"{out.actions[-1].fit_mode}\".")
    ld.sd.name = desc.get("Name", "scene")
    return out


def write_pfm(path: str, rgb: np.ndarray) -> int:
    """Writes an (H, W, 3) float image as a little-endian PFM (rows bottom to top).  Pixels that are not finite or
    have a negative channel are written as (1, 0, 0), as the reference's writer does (PiperRenderer.cpp:272-283);
    returns how many there were."""
    img = np.ascontiguousarray(rgb, dtype=np.float32).copy()
    bad = ~np.all(np.isfinite(img), axis=2) | (np.min(img, axis=2) < 0)
    img[bad] = (1.0, 0.0, 0.0)
    h, w = img.shape[:2]
    with open(path, "wb") as fh:
        fh.write(f"PF\n{w} {h}\n-1.0\n".encode())
        fh.write(img[::-1].astype("<f4").tobytes())
    return int(bad.sum())


def read_pfm(path: str) -> np.ndarray:
    with open(path, "rb") as fh:
        if fh.readline().strip() != b"PF":
            raise ValueError(f"{path}: not a colour PFM")
        w, h = (int(x) for x in fh.readline().split())
        scale = float(fh.readline())
        data = np.frombuffer(fh.read(), dtype="<f4" if scale < 0 else ">f4", count=w * h * 3)
    return data.reshape(h, w, 3)[::-1].astype(np.float32)


def render(options: dict) -> list:
    """Render::execute (PiperRenderer.cpp:306-359): options "ImageSize" [w, h], "SceneDesc" (a JSON path or a
    description), "OutputDir"; "SceneParser" and "Tracer" name the reference's parser and tracer and are not
    used (this library is the tracer).  Renders every action's frames and writes them; returns the written
    paths."""
    from . import api

    size = options.get("ImageSize")
    if not isinstance(size, list) or len(size) != 2:
        raise SceneError("Invalid ImageSize.")
    width, height = int(size[0]), int(size[1])
    scene = load(options["SceneDesc"], options.get("BaseDir"))
    out_dir = options["OutputDir"]
    written = []
    for k, action in enumerate(scene.actions):
        sd = scene.scene_for(action.active_sensor, width, height, action.fit_mode)
        folder = os.path.join(out_dir, f"Action{k}")
        os.makedirs(folder, exist_ok=True)
        with api.Pipeline(sd) as pl:
            for i in range(action.frame_count):
                # every frame renders the sampler's samples of its time interval; nothing moves, so the
                # interval [begin, begin + open) changes no ray (PiperRenderer.cpp:338-345)
                film = pl.new_film()
                pl.launch(film)
                rgb = pl.resolve(film).cpu().numpy()
                path = os.path.join(folder, f"Frame{i}.pfm")
                if write_pfm(path, rgb):
                    warnings.warn("Some invalid pixels are detected.")
                written.append(path)
    return written


def main(argv=None):
    """python -m piper2_b200.scene_json OPTIONS.json: the reference CLI's Render operator over an options file."""
    import sys

    args = sys.argv[1:] if argv is None else argv
    if len(args) != 1:
        print("usage: python -m piper2_b200.scene_json OPTIONS.json", file=sys.stderr)
        return 2
    with open(args[0]) as fh:
        opts = json.load(fh)
    base = os.path.dirname(os.path.abspath(args[0]))
    if isinstance(opts.get("SceneDesc"), str) and not os.path.isabs(opts["SceneDesc"]):
        opts["SceneDesc"] = os.path.join(base, opts["SceneDesc"])
    if not os.path.isabs(opts.get("OutputDir", ".")):
        opts["OutputDir"] = os.path.join(base, opts["OutputDir"])
    for p in render(opts):
        print(p)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
