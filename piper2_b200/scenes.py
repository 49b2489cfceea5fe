"""Seeded synthetic workloads: the scenes, ray sets and render settings of the benchmark configurations.

No scene files are read: every configuration is generated from a seed with numpy's PCG64 generator,
so the same seed gives the same float32 arrays on every machine.

* :func:`cornell_box`        -- the small Cornell-box-style scene (10 + 24 triangles, 0.25 x 0.25
  ceiling light of radiance (17, 12, 4), Lambertian white/red/green, pinhole 40 degree FOV, 256 x 256,
  16 spp, max depth 8, NEE + MIS).
* :func:`triangle_soup` / :func:`soup_rays` -- the traversal stress test: 1M triangles with centroids
  uniform in [0,1]^3 and lognormal edge lengths (median 0.01, sigma 0.5); 4M closest-hit rays from
  the bounding sphere towards uniform interior points, 4M any-hit rays of length U[0.1, 1].

The benchmark scenes bake rotations into vertex positions and use translation-only instances, the only
instance transforms the reference renders correctly (it inverts them with a routine that is only correct for
translations, Src/Kernel/Transform.hpp:344-362).  A mesh may instead carry a full SRT instance transform
(:func:`srt_matrix`, ``MeshData.transform``), which the library flattens into world space when it builds the
acceleration structure -- a divergence from the reference for rotated or scaled instances.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import capi

f32 = np.float32


def plane_make(origin, u, v) -> capi.Plane:
    """PerPlaneData from Origin/U/V exactly as the Plane geometry builds it
    (Src/BuiltinComponent/Geometry/BasicShapes/BasicShapes.cpp:70-89), in float32."""
    o = [f32(x) for x in origin]
    u = [f32(x) for x in u]
    v = [f32(x) for x in v]
    det = [u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]]
    area = np.sqrt(max(det[0] * det[0] + det[1] * det[1] + det[2] * det[2], f32(0)))
    n = [d / area for d in det]
    ul = np.sqrt(max(u[0] * u[0] + u[1] * u[1] + u[2] * u[2], f32(0)))
    t = [x / ul for x in u]
    a = [abs(d) for d in det]
    if a[0] >= a[1] and a[0] >= a[2]:
        sel = 0
    else:
        sel = 1 if (a[1] >= a[0] and a[1] >= a[2]) else 2
    p = capi.Plane()
    p.origin[:] = [float(x) for x in o]
    p.u[:] = [float(x) for x in u]
    p.v[:] = [float(x) for x in v]
    p.normal[:] = [float(x) for x in n]
    p.tangent[:] = [float(x) for x in t]
    p.max_det_comp = sel
    return p


def euler_quaternion(pitch: float, yaw: float, roll: float) -> tuple:
    """The quaternion (w, x, y, z) of the reference's three-angle "Rotation" (Src/PiperRenderer.cpp:113-124), in
    float32 arithmetic."""
    hp, hy, hr = f32(0.5) * f32(pitch), f32(0.5) * f32(yaw), f32(0.5) * f32(roll)
    cp, sp = f32(np.cos(hp)), f32(np.sin(hp))
    cy, sy = f32(np.cos(hy)), f32(np.sin(hy))
    cr, sr = f32(np.cos(hr)), f32(np.sin(hr))
    return (float(cr * cp * cy + sr * sp * sy), float(cr * sp * cy + sr * cp * sy),
            float(cr * cp * sy - sr * sp * cy), float(sr * cp * cy - cr * sp * sy))


def srt(translation=(0.0, 0.0, 0.0), scale=(1.0, 1.0, 1.0), quat=(1.0, 0.0, 0.0, 0.0), skew=(0.0, 0.0, 0.0),
        shift=(0.0, 0.0, 0.0)) -> capi.SRT:
    t = capi.SRT()
    sc = [scale] * 3 if np.isscalar(scale) else list(scale)
    t.scale[:] = [float(x) for x in sc]
    t.skew[:] = [float(x) for x in skew]
    t.shift[:] = [float(x) for x in shift]
    t.quat[:] = [float(x) for x in quat]
    t.translation[:] = [float(x) for x in translation]
    return t


def srt_matrix(transform: capi.SRT | None = None, **kw) -> np.ndarray:
    """The (12,) float32 row-major 3x4 local-to-world matrix of an SRT transform (pb2_srt_matrix); keyword
    arguments build the SRT as :func:`srt` does."""
    t = transform if transform is not None else srt(**kw)
    m = np.zeros(12, np.float32)
    capi.check(capi.lib().pb2_srt_matrix(C.byref(t), m.ctypes.data_as(C.POINTER(C.c_float))))
    return m


def plane_transform(plane: capi.Plane, matrix) -> capi.Plane:
    m = np.ascontiguousarray(matrix, dtype=np.float32).reshape(12)
    out = capi.Plane()
    capi.check(capi.lib().pb2_plane_transform(C.byref(plane), m.ctypes.data_as(C.POINTER(C.c_float)), C.byref(out)))
    return out


def camera_from_config(position, look_at, up, sensor_size_mm, focal_length_mm, fstop) -> capi.Camera:
    """PerspectiveCamera config keys -> camera payload (PerspectiveCamera.cpp:39-44): sizes in mm
    times 1e-3f, up normalised, aperture radius = focal / (2 FStop)."""
    cam = capi.Camera()
    cam.position[:] = [float(f32(x)) for x in position]
    cam.look_at[:] = [float(f32(x)) for x in look_at]
    upv = [f32(x) for x in up]
    ul = np.sqrt(max(upv[0] * upv[0] + upv[1] * upv[1] + upv[2] * upv[2], f32(0)))
    cam.up[:] = [float(x / ul) for x in upv]
    cam.sensor_size[:] = [float(f32(sensor_size_mm[0]) * f32(1e-3)), float(f32(sensor_size_mm[1]) * f32(1e-3))]
    focal = f32(focal_length_mm) * f32(1e-3)
    cam.focal_length = float(focal)
    cam.aperture_radius = float(focal / (f32(2.0) * f32(fstop)))
    return cam


@dataclass
class MeshData:
    vertices: np.ndarray  # (V, 3) float32
    indices: np.ndarray   # (T, 3) uint32
    material: int
    translation: tuple = (0.0, 0.0, 0.0)
    transform: np.ndarray | None = None  # (12,) float32 row-major 3x4 local-to-world, or None
    texcoords: np.ndarray | None = None  # (V, 2) float32, or None


@dataclass
class TextureData:
    """A pb2_texture: an image (texels (H, W, C) uint8, C in 1, 2, 4) or a checkerboard."""
    kind: int
    channel: int
    texels: np.ndarray | None = None
    wrap: int = 0
    scale: float = 1.0
    black: tuple = (0.0, 0.0, 0.0, 0.0)
    white: tuple = (1.0, 1.0, 1.0, 1.0)


def image_texture(texels, wrap: str = "Repeat") -> TextureData:
    t = np.ascontiguousarray(texels, dtype=np.uint8)
    if t.ndim == 2:
        t = t[:, :, None]
    if t.shape[2] == 3:  # RGB is loaded as RGBA (SampledTexture.cpp:133-138)
        t = np.concatenate([t, np.full(t.shape[:2] + (1,), 255, np.uint8)], axis=2)
    if t.shape[2] not in (1, 2, 4):
        raise ValueError("an image texture has 1, 2, 3 or 4 channels")
    return TextureData(capi.TEXTURE_IMAGE, int(t.shape[2]), t, capi.WRAP[wrap])


def checkerboard(scale: float, black, white) -> TextureData:
    if len(black) != len(white) or len(black) not in (1, 2, 4):
        raise ValueError("black and white have the same 1, 2 or 4 channels")
    return TextureData(capi.TEXTURE_CHECKERBOARD, len(black), None, 0, scale, tuple(black), tuple(white))


@dataclass
class SceneData:
    meshes: list = field(default_factory=list)
    planes: list = field(default_factory=list)        # capi.Plane
    area_lights: list = field(default_factory=list)   # (radiance, first_plane, plane_count, translation)
    materials: list = field(default_factory=list)     # capi.Material
    textures: list = field(default_factory=list)      # TextureData; material.texture[k] = 1 + index
    env_radiance: tuple = (0.0, 0.0, 0.0)
    settings: capi.RenderSettings | None = None
    name: str = ""

    @property
    def triangle_count(self) -> int:
        return int(sum(m.indices.shape[0] for m in self.meshes))

    def to_ctypes(self):
        """Returns (capi.Scene, keepalive) -- keep the second value alive while the struct is used."""
        keep = []
        meshes = (capi.Mesh * max(1, len(self.meshes)))()
        for i, m in enumerate(self.meshes):
            v = np.ascontiguousarray(m.vertices, dtype=np.float32)
            ix = np.ascontiguousarray(m.indices, dtype=np.uint32)
            keep += [v, ix]
            meshes[i].vertices = v.ctypes.data
            meshes[i].indices = ix.ctypes.data
            meshes[i].texcoords = None
            meshes[i].vert_count = v.shape[0]
            meshes[i].tri_count = ix.shape[0]
            meshes[i].material = m.material
            meshes[i].translation[:] = [float(x) for x in m.translation]
            if m.texcoords is not None:
                tc = np.ascontiguousarray(m.texcoords, dtype=np.float32).reshape(-1, 2)
                if tc.shape[0] != v.shape[0]:
                    raise ValueError("texcoords must hold one (u, v) per vertex")
                keep.append(tc)
                meshes[i].texcoords = tc.ctypes.data
            if m.transform is not None:
                t = np.ascontiguousarray(m.transform, dtype=np.float32).reshape(12)
                keep.append(t)
                meshes[i].transform = t.ctypes.data
            else:
                meshes[i].transform = None
        planes = (capi.Plane * max(1, len(self.planes)))(*self.planes)
        lights = (capi.AreaLight * max(1, len(self.area_lights)))()
        for i, (rad, first, count, tr) in enumerate(self.area_lights):
            lights[i].radiance[:] = [float(x) for x in rad]
            lights[i].first_plane = first
            lights[i].plane_count = count
            lights[i].translation[:] = [float(x) for x in tr]
        mats = (capi.Material * max(1, len(self.materials)))(*self.materials)
        sc = capi.Scene()
        sc.meshes = C.cast(meshes, C.POINTER(capi.Mesh))
        sc.mesh_count = len(self.meshes)
        sc.planes = C.cast(planes, C.POINTER(capi.Plane))
        sc.plane_count = len(self.planes)
        sc.area_lights = C.cast(lights, C.POINTER(capi.AreaLight))
        sc.area_light_count = len(self.area_lights)
        sc.materials = C.cast(mats, C.POINTER(capi.Material))
        sc.material_count = len(self.materials)
        sc.env_radiance[:] = [float(x) for x in self.env_radiance]
        texs = (capi.Texture * max(1, len(self.textures)))()
        for i, t in enumerate(self.textures):
            texs[i].kind, texs[i].channel, texs[i].wrap = t.kind, t.channel, t.wrap
            if t.texels is not None:
                tx = np.ascontiguousarray(t.texels, dtype=np.uint8)
                keep.append(tx)
                texs[i].height, texs[i].width = tx.shape[0], tx.shape[1]
                texs[i].texels = tx.ctypes.data
            texs[i].scale = float(t.scale)
            texs[i].black[:] = [float(x) for x in list(t.black) + [0.0] * (4 - len(t.black))]
            texs[i].white[:] = [float(x) for x in list(t.white) + [0.0] * (4 - len(t.white))]
        sc.textures = C.cast(texs, C.POINTER(capi.Texture))
        sc.texture_count = len(self.textures)
        keep += [meshes, planes, lights, mats, texs]
        return sc, keep


def material(kind: str, color0=(0, 0, 0, 0), color1=(0, 0, 0, 0), roughness=(0.0, 0.0),
             textures=(0, 0, 0, 0)) -> capi.Material:
    """`textures`: per (color0, color1, roughness[0], roughness[1]), 0 or 1 + an index into SceneData.textures."""
    m = capi.Material()
    m.texture[:] = [int(x) for x in textures]
    m.type = capi.SURFACE[kind]
    c0 = list(color0) + [0.0] * (4 - len(color0))
    c1 = list(color1) + [0.0] * (4 - len(color1))
    m.color0[:] = [float(x) for x in c0]
    m.color1[:] = [float(x) for x in c1]
    m.roughness[:] = [float(x) for x in roughness]
    return m


def _quad(p0, p1, p2, p3):
    v = np.array([p0, p1, p2, p3], dtype=np.float64)
    ix = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32)
    return v, ix


def _box(center, size, angle):
    """Axis-aligned box of `size` rotated about +Y by `angle` (radians), resting on y = center[1]."""
    sx, sy, sz = size
    corners = np.array([[x, y, z] for y in (0.0, sy) for z in (-sz / 2, sz / 2) for x in (-sx / 2, sx / 2)])
    c, s = math.cos(angle), math.sin(angle)
    rot = np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])
    v = corners @ rot.T + np.array(center)
    # corner index = y*4 + z*2 + x
    faces = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    ix = []
    for a, b, cc, d in faces:
        ix += [[a, b, cc], [a, cc, d]]
    return v, np.array(ix, dtype=np.uint32)


def render_settings(width, height, spp, max_depth, min_rr_depth, camera, filt="box", alpha=2.0,
                    fit="Fill", scramble=0, scramble_seed=0) -> capi.RenderSettings:
    st = capi.RenderSettings()
    st.width, st.height = width, height
    st.fit_mode = capi.FIT[fit]
    if spp & (spp - 1):
        spp = 1 << int(math.ceil(math.log2(spp)))  # ScrambledSobolSampler.cpp:43-50
    st.samples_per_pixel = spp
    st.scramble = scramble  # 1: Owen scrambling of dimensions >= 2 (extension; the reference has none)
    st.scramble_seed = scramble_seed
    st.max_depth = max_depth
    st.min_rr_depth = min_rr_depth
    st.filter = capi.FILTER[filt]
    st.gaussian_alpha = alpha
    st.camera = camera
    return st


def cornell_box(seed: int = 0, width: int = 256, height: int = 256, spp: int = 16, max_depth: int = 8,
                min_rr_depth: int = 3) -> SceneData:
    rng = np.random.default_rng(seed)
    a1, a2 = np.deg2rad(rng.uniform(-30.0, 30.0, size=2))
    white, red, green = 0, 1, 2
    sd = SceneData(name=f"cornell_box(seed={seed})")
    sd.materials = [material("Matte", (0.73, 0.73, 0.73, 1.0)),
                    material("Matte", (0.65, 0.05, 0.05, 1.0)),
                    material("Matte", (0.12, 0.45, 0.15, 1.0))]
    room = [
        (_quad((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1)), white),   # floor
        (_quad((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0)), white),   # ceiling
        (_quad((0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)), white),   # back wall
        (_quad((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1)), red),     # x = 1 wall (left in the image)
        (_quad((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0)), green),   # x = 0 wall (right in the image)
    ]
    for (v, ix), mat in room:
        sd.meshes.append(MeshData(v.astype(np.float32), ix, mat))
    for center, size, ang in (((0.68, 0.0, 0.35), (0.28, 0.28, 0.28), a1),
                              ((0.33, 0.0, 0.65), (0.28, 0.56, 0.28), a2)):
        v, ix = _box(center, size, ang)
        sd.meshes.append(MeshData(v.astype(np.float32), ix, white))
    sd.planes = [plane_make((0.375, 0.999, 0.375), (0.25, 0.0, 0.0), (0.0, 0.0, 0.25))]
    sd.area_lights = [((17.0, 12.0, 4.0), 0, 1, (0.0, 0.0, 0.0))]
    sd.env_radiance = (0.0, 0.0, 0.0)  # the pipeline requires one infinite light (Embree.cpp:1185-1188)
    focal_mm = 35.0
    sensor_mm = 2.0 * focal_mm * math.tan(math.radians(20.0))  # 40 degree field of view
    cam = camera_from_config((0.5, 0.5, -1.4), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0), (sensor_mm, sensor_mm), focal_mm,
                             1e30)
    sd.settings = render_settings(width, height, spp, max_depth, min_rr_depth, cam)
    return sd


def _unit_cube():
    """The cube [-0.5, 0.5] x [0, 1] x [-0.5, 0.5] (12 triangles, outward winding as :func:`_box`)."""
    return _box((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 0.0)


def instanced_room(seed: int = 0, width: int = 64, height: int = 64, spp: int = 8, max_depth: int = 8,
                   min_rr_depth: int = 3, light_tilt: float = 0.35) -> SceneData:
    """The Cornell room with its boxes as instances of one unit cube under full SRT transforms (scale, a
    rotation about a tilted axis, skew, translation) and the ceiling light tilted by `light_tilt` radians about
    the x axis through its centre: geometry the reference can only render correctly with rotations baked into the
    vertices.  Materials: white Matte walls, a Plastic box and a rough Glass box."""
    rng = np.random.default_rng(seed)
    sd = cornell_box(seed=seed, width=width, height=height, spp=spp, max_depth=max_depth, min_rr_depth=min_rr_depth)
    sd.name = f"instanced_room(seed={seed})"
    sd.meshes = sd.meshes[:5]
    sd.materials.append(material("Plastic", (0.4, 0.3, 0.6), (0.5, 0.5, 0.5), (0.25, 0.0)))
    sd.materials.append(material("Glass", (1, 1, 1), (1, 1, 1), (0.15, 0.15)))
    v, ix = _unit_cube()
    v = v.astype(np.float32)
    for k, (center, size) in enumerate((((0.68, 0.0, 0.35), (0.28, 0.28, 0.28)),
                                        ((0.33, 0.02, 0.65), (0.26, 0.5, 0.22)))):
        axis = rng.normal(size=3) * (0.3, 1.0, 0.3)
        axis /= np.linalg.norm(axis)
        ang = rng.uniform(-0.6, 0.6)
        q = (math.cos(ang / 2), *(math.sin(ang / 2) * axis))
        skew = (rng.uniform(-0.1, 0.1), 0.0, rng.uniform(-0.1, 0.1))
        m = srt_matrix(translation=center, scale=size, quat=q, skew=skew)
        sd.meshes.append(MeshData(v, ix, 3 + k, transform=m))
    c = np.array([0.5, 0.95, 0.5], np.float32)
    light = plane_make((0.375, 0.95, 0.375), (0.25, 0.0, 0.0), (0.0, 0.0, 0.25))
    # rotate about the x axis through the light's centre: T(c) R T(-c)
    qa = (math.cos(light_tilt / 2), math.sin(light_tilt / 2), 0.0, 0.0)
    r = srt_matrix(quat=qa).reshape(3, 4)
    t = c - r[:, :3] @ c
    m = np.concatenate([r[:, :3], t[:, None].astype(np.float32)], axis=1).astype(np.float32)
    sd.planes = [plane_transform(light, m)]
    return sd


def textured_room(seed: int = 0, width: int = 48, height: int = 48, spp: int = 8, max_depth: int = 8,
                  min_rr_depth: int = 3) -> SceneData:
    """The Cornell room with textured materials: a checkerboard floor, an RGB image on the back wall (texcoords
    running past [0, 1], wrap Repeat), a Plastic box whose roughness is a grey image (wrap Mirror) and a Substrate
    box with a roughness checkerboard, plus a textured material on a mesh without texcoords (which samples at
    (0, 0)).  Images are seeded noise, 8-bit."""
    rng = np.random.default_rng(seed)
    sd = cornell_box(seed=seed, width=width, height=height, spp=spp, max_depth=max_depth, min_rr_depth=min_rr_depth)
    sd.name = f"textured_room(seed={seed})"
    img = rng.integers(0, 256, size=(13, 17, 3), dtype=np.uint8)
    grey = rng.integers(0, 256, size=(9, 7), dtype=np.uint8)
    sd.textures = [checkerboard(6.0, (0.1, 0.1, 0.1, 1.0), (0.8, 0.75, 0.7, 1.0)),  # 1: floor color
                   image_texture(img, "Repeat"),                                   # 2: back wall color
                   image_texture(grey, "Mirror"),                                  # 3: plastic roughness
                   checkerboard(3.0, (0.05,), (0.6,)),                             # 4: substrate roughness x
                   image_texture(grey[::-1].copy(), "Repeat")]                     # 5: substrate roughness y
    sd.materials += [material("Matte", (0, 0, 0), textures=(1, 0, 0, 0)),
                     material("Matte", (0, 0, 0), textures=(2, 0, 0, 0)),
                     material("Plastic", (0.3, 0.4, 0.6), (0.5, 0.5, 0.5), (0.2, 0.0), textures=(0, 0, 3, 0)),
                     material("Substrate", (0.5, 0.3, 0.2), (0.3, 0.3, 0.3), (0.1, 0.1), textures=(0, 0, 4, 5))]
    sd.meshes[0].material = 3       # floor
    sd.meshes[0].texcoords = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    sd.meshes[2].material = 4       # back wall
    sd.meshes[2].texcoords = np.array([[-0.3, 0.1], [2.2, 0.1], [2.2, 1.7], [-0.3, 1.7]], np.float32)
    sd.meshes[1].material = 3       # ceiling: textured material, no texcoords
    for k, m in ((5, 5), (6, 6)):
        sd.meshes[k].material = m
        n = sd.meshes[k].vertices.shape[0]
        sd.meshes[k].texcoords = rng.uniform(-1.5, 2.5, size=(n, 2)).astype(np.float32)
    return sd


def triangle_soup(n_tris: int = 1 << 20, seed: int = 0) -> SceneData:
    """Traversal stress scene: centroids U[0,1]^3, vertices at lognormal distance (median 0.01,
    sigma 0.5) from the centroid along random unit directions."""
    rng = np.random.default_rng(seed)
    cen = rng.random((n_tris, 1, 3))
    scale = np.exp(rng.normal(math.log(0.01), 0.5, size=(n_tris, 1, 1)))
    d = rng.normal(size=(n_tris, 3, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    v = (cen + scale * d).reshape(-1, 3).astype(np.float32)
    ix = np.arange(3 * n_tris, dtype=np.uint32).reshape(n_tris, 3)
    sd = SceneData(name=f"triangle_soup(n={n_tris}, seed={seed})")
    sd.materials = [material("Matte", (0.5, 0.5, 0.5, 1.0))]
    sd.meshes = [MeshData(v, ix, 0)]
    return sd


def soup_rays(n_rays: int = 1 << 22, seed: int = 1, kind: str = "closest") -> np.ndarray:
    """Ray sets of the traversal stress test, as a RAY_DTYPE array.

    closest: origin uniform on the sphere around [0,1]^3 (centre 0.5, radius sqrt(3)/2 + 0.01), direction
    towards a uniform point of [0,1]^3, t in (0, 1e30).  any: origin uniform in [0,1]^3, uniform
    direction, t in (0, U[0.1, 1])."""
    rng = np.random.default_rng(seed)
    rays = np.zeros(n_rays, dtype=capi.RAY_DTYPE)
    if kind == "closest":
        s = rng.normal(size=(n_rays, 3))
        s /= np.linalg.norm(s, axis=1, keepdims=True)
        org = 0.5 + (math.sqrt(3.0) / 2 + 0.01) * s
        tgt = rng.random((n_rays, 3))
        d = tgt - org
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        rays["tmax"] = 1e30
    else:
        org = rng.random((n_rays, 3))
        d = rng.normal(size=(n_rays, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        rays["tmax"] = rng.uniform(0.1, 1.0, size=n_rays)
    rays["org"] = org
    rays["dir"] = d
    rays["tmin"] = 0.0
    return rays


def _grid_quad(origin, u, v, nu, nv):
    """Quad origin + [0,1]u + [0,1]v tessellated into nu x nv cells (2 triangles each)."""
    o, u, v = (np.asarray(x, dtype=np.float64) for x in (origin, u, v))
    a = np.linspace(0.0, 1.0, nu + 1)
    b = np.linspace(0.0, 1.0, nv + 1)
    A, B = np.meshgrid(a, b, indexing="ij")
    verts = o + A[..., None] * u + B[..., None] * v
    verts = verts.reshape(-1, 3)
    idx = []
    for i in range(nu):
        for j in range(nv):
            p00 = i * (nv + 1) + j
            p10 = (i + 1) * (nv + 1) + j
            p01 = p00 + 1
            p11 = p10 + 1
            idx += [[p00, p10, p11], [p00, p11, p01]]
    return verts, np.array(idx, dtype=np.uint32)


def guiding_room(seed: int = 0, width: int = 1280, height: int = 720, spp: int = 256, max_depth: int = 16,
                 min_rr_depth: int = 5, tess: int = 15) -> SceneData:
    """Hard indirect lighting: a 4 x 2.5 x 4 m room split by a wall at x = 2.5 with a 5 cm door gap; the only
    area light (0.1 m^2, radiance 200) hangs behind the wall; the floor of the camera's side is glossy GGX
    (alpha 0.1, the conductor extension); white Lambertian walls.  About 20k triangles (every quad is
    tessellated)."""
    rng = np.random.default_rng(seed)
    sd = SceneData(name=f"guiding_room(seed={seed})")
    white, floor = 0, 1
    sd.materials = [material("Matte", (0.75, 0.75, 0.75, 1.0)),
                    material("Conductor", color1=(0.9, 0.85, 0.8, 1.0), roughness=(0.1, 0.1))]
    W, H, D = 4.0, 2.5, 4.0
    xw = 2.5                                      # dividing wall
    gap_z0, gap_z1, gap_h = 1.975, 2.025, 2.0     # 5 cm wide, 2 m tall door gap
    quads = [
        ((0, 0, 0), (xw, 0, 0), (0, 0, D), floor),            # glossy floor, camera side
        ((xw, 0, 0), (W - xw, 0, 0), (0, 0, D), white),        # floor behind the wall
        ((0, H, 0), (0, 0, D), (W, 0, 0), white),              # ceiling
        ((0, 0, 0), (0, H, 0), (0, 0, D), white),              # x = 0 wall
        ((W, 0, 0), (0, 0, D), (0, H, 0), white),              # x = W wall
        ((0, 0, 0), (W, 0, 0), (0, H, 0), white),              # z = 0 wall
        ((0, 0, D), (0, H, 0), (W, 0, 0), white),              # z = D wall
        # dividing wall at x = xw: left of the gap, right of the gap, above the gap
        ((xw, 0, 0), (0, 0, gap_z0), (0, H, 0), white),
        ((xw, 0, gap_z1), (0, 0, D - gap_z1), (0, H, 0), white),
        ((xw, gap_h, gap_z0), (0, 0, gap_z1 - gap_z0), (0, H - gap_h, 0), white),
    ]
    for o, u, v, mat in quads:
        nu = max(1, int(round(tess * np.linalg.norm(u) / 4.0 * 3)))
        nv = max(1, int(round(tess * np.linalg.norm(v) / 4.0 * 3)))
        verts, ix = _grid_quad(o, u, v, nu, nv)
        sd.meshes.append(MeshData(verts.astype(np.float32), ix, mat))
    # a few seed-placed boxes in the camera's room
    for _ in range(3):
        c = (rng.uniform(0.4, 2.0), 0.0, rng.uniform(0.5, 3.5))
        s = (rng.uniform(0.2, 0.5), rng.uniform(0.3, 0.9), rng.uniform(0.2, 0.5))
        v, ix = _box(c, s, rng.uniform(-0.5, 0.5))
        sd.meshes.append(MeshData(v.astype(np.float32), ix, white))
    side = float(np.sqrt(0.1))
    sd.planes = [plane_make((3.25 - side / 2, 2.45, 2.0 - side / 2), (side, 0.0, 0.0), (0.0, 0.0, side))]
    sd.area_lights = [((200.0, 200.0, 200.0), 0, 1, (0.0, 0.0, 0.0))]
    sd.env_radiance = (0.0, 0.0, 0.0)
    cam = camera_from_config((0.15, 1.3, 0.25), (2.5, 1.0, 2.2), (0.0, 1.0, 0.0), (36.0, 20.25), 24.0, 1e30)
    sd.settings = render_settings(width, height, spp, max_depth, min_rr_depth, cam)
    return sd


def _icosphere(subdiv: int):
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    for _ in range(subdiv):
        cache = {}
        nf = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return np.array(verts), np.array(f, dtype=np.uint32)


def _fbm(x, z, rng_offsets, octaves=6):
    h = np.zeros_like(x)
    amp, freq = 0.5, 1.0
    for o in range(octaves):
        ox, oz, ph = rng_offsets[o]
        h += amp * np.sin(freq * 2.1 * x + ox) * np.cos(freq * 1.7 * z + oz) + amp * 0.5 * np.sin(freq * 3.3 * (x + z) + ph)
        amp *= 0.5
        freq *= 2.0
    return h


def mixed_materials(seed: int = 0, width: int = 1920, height: int = 1080, spp: int = 64, max_depth: int = 16,
                    min_rr_depth: int = 5, grid: int = 1024, n_spheres: int = 200) -> SceneData:
    """Mixed-material scene: a grid x grid heightfield terrain (2 grid^2 triangles) from 6-octave fBm, with
    n_spheres translated subdivision-4 icospheres (5120 triangles each) whose material is drawn per sphere:
    GGX conductor (alpha U[0.05, 0.5]), smooth dielectric (IOR 1.5, the reference's Glass) or Lambert
    (albedo U[0.1, 0.9]).  Constant environment 0.5 and one small sun-like area light."""
    rng = np.random.default_rng(seed)
    sd = SceneData(name=f"mixed_materials(seed={seed})")
    sd.materials = [material("Matte", (0.35, 0.32, 0.28, 1.0))]
    size = 40.0
    xs = np.linspace(-size / 2, size / 2, grid + 1)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    offs = rng.uniform(0, 6.28, size=(6, 3))
    Y = 1.5 * _fbm(X / 8.0, Z / 8.0, offs)
    verts = np.stack([X, Y, Z], axis=-1).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(grid), np.arange(grid), indexing="ij")
    p00 = (i * (grid + 1) + j).ravel()
    p10 = p00 + (grid + 1)
    ix = np.stack([np.stack([p00, p10 + 1, p10], 1), np.stack([p00, p00 + 1, p10 + 1], 1)], 1).reshape(-1, 3)
    sd.meshes.append(MeshData(verts.astype(np.float32), ix.astype(np.uint32), 0))
    sv, sf = _icosphere(4)
    for k in range(n_spheres):
        r = rng.uniform(0.3, 1.0)
        px, pz = rng.uniform(-size / 2.5, size / 2.5, size=2)
        py = float(1.5 * _fbm(np.array([px / 8.0]), np.array([pz / 8.0]), offs)[0]) + r
        kind = rng.integers(0, 3)
        if kind == 0:
            a = rng.uniform(0.05, 0.5)
            sd.materials.append(material("Conductor", color1=tuple(rng.uniform(0.5, 0.95, 3)) + (1.0,), roughness=(a, a)))
        elif kind == 1:
            sd.materials.append(material("Glass", (1, 1, 1, 1), (1, 1, 1, 1), (0.0, 0.0)))
        else:
            alb = rng.uniform(0.1, 0.9)
            sd.materials.append(material("Matte", (alb, alb * rng.uniform(0.6, 1.0), alb * rng.uniform(0.6, 1.0), 1.0)))
        sd.meshes.append(MeshData((sv * r).astype(np.float32), sf, len(sd.materials) - 1, (float(px), py, float(pz))))
    sd.planes = [plane_make((-2.0, 30.0, -2.0), (4.0, 0.0, 0.0), (0.0, 0.0, 4.0))]
    sd.area_lights = [((400.0, 380.0, 340.0), 0, 1, (0.0, 0.0, 0.0))]
    sd.env_radiance = (0.5, 0.5, 0.5)
    cam = camera_from_config((0.0, 8.0, -24.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), (36.0, 20.25), 28.0, 1e30)
    sd.settings = render_settings(width, height, spp, max_depth, min_rr_depth, cam)
    return sd


def _grid_cells(p0, p1, p3, n):
    """The parallelogram p0 + [0,1](p1 - p0) + [0,1](p3 - p0) as an n x n grid of cells, two triangles each, wound
    as the quad [p0, p1, p2], [p0, p2, p3] (vectorised)."""
    p0, p1, p3 = (np.asarray(x, dtype=np.float64) for x in (p0, p1, p3))
    a = np.linspace(0.0, 1.0, n + 1)
    A, B = np.meshgrid(a, a, indexing="ij")
    verts = (p0 + A[..., None] * (p1 - p0) + B[..., None] * (p3 - p0)).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    p00 = (i * (n + 1) + j).reshape(-1)
    p10, p01 = p00 + (n + 1), p00 + 1
    p11 = p10 + 1
    idx = np.stack([np.stack([p00, p10, p11], 1), np.stack([p00, p11, p01], 1)], 1).reshape(-1, 3)
    return verts, idx.astype(np.uint32)


def cornell_variant(seed: int = 0, triangles: int = 10_000, width: int = 256, height: int = 256, spp: int = 16,
                    max_depth: int = 16, min_rr_depth: int = 3) -> SceneData:
    """A variant of the Cornell-box generator with about `triangles` triangles: the seed draws the boxes' angles
    as :func:`cornell_box` does, and the five room quads are tessellated into equal grids (same surfaces, same
    image, more geometry to traverse)."""
    sd = cornell_box(seed=seed, width=width, height=height, spp=spp, max_depth=max_depth, min_rr_depth=min_rr_depth)
    n = max(1, int(np.sqrt(max(triangles - 24, 10) / 10)))
    for m in sd.meshes[:5]:
        v = m.vertices.astype(np.float64)
        gv, gi = _grid_cells(v[0], v[1], v[3], n)
        m.vertices, m.indices = gv.astype(np.float32), gi
    sd.name = f"cornell_variant(seed={seed}, {sd.triangle_count} tris)"
    return sd


def batch_workload(seed: int = 0, count: int = 64, max_depth: int = 16) -> list:
    """The batching workload: `count` scenes, each a seed-drawn variant of the Cornell-box generator
    (:func:`cornell_variant`) or of the mixed-materials generator (:func:`mixed_materials`), chosen with equal
    probability, with its own seed, a triangle count log-uniform in [10k, 2M] (room grid, or terrain grid and
    icosphere count, chosen to match), film side log-uniform in [128, 1024] (16:9), and spp uniform in [4, 64]
    rounded up to a power of two (the reference's sampler rounds the same way,
    ScrambledSobolSampler.cpp:43-50)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        tris = int(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        side = int(np.exp(rng.uniform(np.log(128), np.log(1024))))
        width, height = side, max(8, int(round(side * 9 / 16)))
        spp = 1 << int(np.ceil(np.log2(rng.integers(4, 65))))
        if rng.uniform() < 0.5:
            sd = cornell_variant(seed=seed * 1000 + k + 1, triangles=tris, width=width, height=height, spp=spp,
                                 max_depth=max_depth)
            sd.name = f"batch[{k}] cornell {sd.triangle_count} tris {width}x{height} {spp} spp"
        else:
            n_spheres = int(min(200, (0.3 * tris) // 5120))
            grid = max(8, int(np.sqrt(max(tris - 5120 * n_spheres, 128) / 2)))
            sd = mixed_materials(seed=seed * 1000 + k + 1, width=width, height=height, spp=spp, max_depth=max_depth,
                                 grid=grid, n_spheres=n_spheres)
            sd.name = f"batch[{k}] mixed {2 * grid * grid + 5120 * n_spheres} tris {width}x{height} {spp} spp"
        out.append(sd)
    return out

