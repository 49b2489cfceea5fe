"""Textures (CheckBoard, Texture/ProceduralTexture/Kernel.cpp:27-38; the bilinear SampledTexture,
Texture/SampledTexture/Kernel.cpp:22-83; texture coordinates of calcTriangleMeshSurface,
Tracer/Embree/Kernel.cpp:181-190) and the per-point roughness remap they need: the shared pb2_math.h definitions
(run by the oracle here and by the device in the GPU tests) against a restatement of the reference's kernels, the
textured room rendered by the oracle against the reference's own kernels compiled natively, and the library's
validation of texture bindings.  Host-side only: runs without a GPU."""
import ctypes as C
import math
import os

import numpy as np
import pytest

from piper2_b200 import capi, scenes

f32 = np.float32
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _ulp_diff(a, b):
    a = np.asarray(a, f32).view(np.int32).astype(np.int64)
    b = np.asarray(b, f32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


def test_logf_within_two_ulp(oracle):
    lib = oracle.oracle()
    rng = np.random.default_rng(0)
    xs = np.concatenate([np.exp(rng.uniform(-87, 88, 20000)), rng.uniform(0.5, 2.0, 5000), [1.0, 2.0, 0.5, 1e-3],
                         [1.4e-40, 3e-39]]).astype(f32)
    got = np.array([lib.or_logf(float(x)) for x in xs], f32)
    exp = np.log(xs.astype(np.float64)).astype(f32)
    assert _ulp_diff(got, exp).max() <= 2


def test_point_remap_matches_the_host_remap(oracle):
    """The polynomial of remapRoughness cancels heavily (terms up to ~8 summing to ~0.2), so a last-bit difference
    of the logarithm shows as an absolute difference of a few 1e-7."""
    lib = oracle.oracle()
    for r in np.linspace(0.0, 1.0, 2001, dtype=f32):
        a, b = lib.or_remap_roughness_point(float(r)), lib.or_remap_roughness(float(r))
        assert abs(a - b) <= 5e-7, r


def _restated_sample(texels, wrap, tu, tv):
    """SampledTexture/Kernel.cpp:22-83 restated in float32 numpy, operation for operation."""
    h, w, ch = texels.shape
    flat = texels.reshape(-1)

    def locate(p, size):
        rem = f32(math.remainder(float(p), float(size)))
        s = (rem + f32(size) if rem < 0 else rem) if wrap == 0 else abs(rem)
        return min(int(s), size - 1)

    def nxt(p, size):
        s = p + 1
        return (0 if wrap == 0 else p) if s == size else s

    u, v = f32(tu) * f32(w), f32(tv) * f32(h)
    plu = locate(u - f32(0.5), w)
    pru = nxt(plu, w)
    plv = locate(v - f32(0.5), h)
    prv = nxt(plv, h)
    lw = lambda x: (f32(0.5) + f32(math.floor(x + f32(0.5)))) - x  # noqa: E731
    lwx, lwy = lw(u), lw(v)
    rwx, rwy = f32(1) - lwx, f32(1) - lwy
    out = np.zeros(ch, f32)
    for cu, cv, wt in ((plu, plv, lwx * lwy), (pru, plv, rwx * lwy), (plu, prv, lwx * rwy), (pru, prv, rwx * rwy)):
        idx = cv * w * ch + cu * ch
        for i in range(ch):
            out[i] = out[i] + wt * f32(flat[idx + i])
    return out * f32(0.003921568)


def _restated_checker(scale, black, white, tu, tv):
    def mod(x):
        r = f32(math.remainder(float(f32(x) * f32(scale)), 2.0))
        return r + f32(2) if r < 0 else r

    return np.array(white if (mod(tu) > 1) == (mod(tv) > 1) else black, f32)


def _ctex(t: scenes.TextureData):
    sd = scenes.SceneData(textures=[t])
    sc, keep = sd.to_ctypes()
    return sc.textures, keep


@pytest.mark.parametrize("channels,wrap", [(4, "Repeat"), (1, "Mirror"), (4, "Mirror"), (2, "Repeat")])
def test_image_sampling_matches_the_reference_kernel(oracle, channels, wrap):
    rng = np.random.default_rng(channels * 7 + len(wrap))
    img = rng.integers(0, 256, size=(11, 6, channels), dtype=np.uint8)
    tex = scenes.image_texture(img, wrap)
    ct, keep = _ctex(tex)
    out = (C.c_float * 4)()
    coords = np.concatenate([rng.uniform(-3, 3, (400, 2)), [[0, 0], [1, 1], [0.5, 0.5], [1 / 12, 1 / 11]]]).astype(f32)
    for tu, tv in coords:
        oracle.oracle().or_texture_sample(ct, float(tu), float(tv), out)
        exp = _restated_sample(img, capi.WRAP[wrap], tu, tv)
        got = np.array(out[:channels], f32)
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), (tu, tv, got, exp)


def test_checkerboard_matches_the_reference_kernel(oracle):
    rng = np.random.default_rng(9)
    tex = scenes.checkerboard(3.7, (0.1, 0.2, 0.3, 1.0), (0.9, 0.8, 0.7, 0.5))
    ct, keep = _ctex(tex)
    out = (C.c_float * 4)()
    for tu, tv in rng.uniform(-4, 4, (500, 2)).astype(f32):
        oracle.oracle().or_texture_sample(ct, float(tu), float(tv), out)
        exp = _restated_checker(3.7, tex.black, tex.white, tu, tv)
        assert np.array_equal(np.array(out[:4], f32), exp)


def test_rgb_images_load_as_rgba():
    t = scenes.image_texture(np.zeros((2, 3, 3), np.uint8))
    assert t.channel == 4 and t.texels.shape == (2, 3, 4) and (t.texels[..., 3] == 255).all()


def _compare(osamp, rsamp):
    assert np.array_equal(osamp[..., :2], rsamp[..., :2]), "film points differ"
    exact = np.all(osamp[..., 2:] == rsamp[..., 2:], axis=-1)
    rel = np.abs(osamp[..., 2:] - rsamp[..., 2:]).max(-1) / (np.abs(rsamp[..., 2:]).max(-1) + 1e-6)
    # differences come from the C library's sin/cos/log against pb2_math's (last bit) on a few paths
    assert exact.mean() > 0.85, exact.mean()
    assert (rel > 1e-3).mean() < 5e-3, (rel > 1e-3).mean()


def test_textured_room_oracle_vs_golden_reference_vectors(oracle):
    """Per-sample radiance of the textured room from the reference's own kernels (tests/golden/make_golden.py)."""
    data = np.load(os.path.join(GOLDEN, "textured_room_32x32_4spp.npz"))
    sd = scenes.textured_room(seed=int(data["seed"]), width=32, height=32, spp=4)
    _, osamp = oracle.OracleScene(sd, use_bvh=False).render(sd.settings)
    _compare(osamp, data["samples"])


def test_textured_room_oracle_vs_reference_kernels(oracle):
    if not oracle.ref_available():
        pytest.skip("reference harness not built")
    sd = scenes.textured_room(seed=3, width=40, height=40, spp=4)
    _, osamp = oracle.OracleScene(sd, use_bvh=True).render(sd.settings)
    _, rsamp = oracle.RefScene(sd, use_bvh=True).render()
    _compare(osamp, rsamp)


def _create_fails(sd, match):
    lib = capi.lib()
    sc, keep = sd.to_ctypes()
    h = C.c_void_p()
    rc = lib.pb2_pipeline_create(C.byref(sc), C.byref(sd.settings), None, C.byref(h))
    assert rc == capi.PB2_ERR_INVALID_ARGUMENT, rc
    assert match in lib.pb2_last_error().decode()


def test_texture_bindings_are_validated():
    sd = scenes.textured_room(seed=0)
    sd.materials[3].texture[0] = 4          # a 1-channel texture bound to a color
    _create_fails(sd, "mismatched channel, expect 4, but get 1")
    sd = scenes.textured_room(seed=0)
    sd.materials[5].texture[2] = 2          # a 4-channel texture bound to a roughness
    _create_fails(sd, "mismatched channel, expect 1, but get 4")
    sd = scenes.textured_room(seed=0)
    sd.materials[3].texture[0] = 9
    _create_fails(sd, "texture index out of range")
    sd = scenes.textured_room(seed=0)
    sd.textures[1].wrap = 5
    _create_fails(sd, "wrap mode")
