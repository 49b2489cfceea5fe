"""Transformed instances on the GPU (a documented divergence from the reference, whose calcInverse,
Src/Kernel/Transform.hpp:344-362, only inverts translations): a room whose boxes are one unit cube under
scale/rotation/skew/translation and whose light is tilted renders every sample bit-exact against the CPU oracle,
exactly as the same room with the transforms baked into the vertices, and its closest hits through the C ABI are
the oracle's."""
import numpy as np
import pytest

from piper2_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def _api():
    from piper2_b200 import api

    return api


def _baked(sd):
    f32 = np.float32
    for m in sd.meshes:
        if m.transform is not None:
            v = m.vertices.astype(f32)
            t = np.asarray(m.transform, f32).reshape(3, 4)
            v = ((t[:, 0] * v[:, :1] + t[:, 1] * v[:, 1:2]) + t[:, 2] * v[:, 2:3]) + t[:, 3]
            m.vertices, m.transform = v + np.asarray(m.translation, f32), None
            m.translation = (0.0, 0.0, 0.0)
    return sd


@pytest.mark.parametrize("seed", [0, 1])
def test_instanced_room_samples_bitexact(oracle, seed):
    sd = scenes.instanced_room(seed=seed, width=48, height=48, spp=8)
    with _api().Pipeline(sd) as pl:
        film, samples = pl.render(samples=True)
    ofilm, osamples = oracle.OracleScene(sd, use_bvh=True).render(sd.settings)
    diff = np.any(samples.view(np.uint32) != osamples.view(np.uint32), axis=-1)
    assert not diff.any(), f"{diff.sum()} of {diff.size} samples differ"
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)
    assert film[..., :3].sum() > 0
    with _api().Pipeline(_baked(scenes.instanced_room(seed=seed, width=48, height=48, spp=8))) as pl:
        _, baked = pl.render(samples=True)
    assert np.array_equal(samples.view(np.uint32), baked.view(np.uint32))


def test_instanced_closest_hits_match_the_oracle(oracle):
    sd = scenes.instanced_room(seed=2)
    rng = np.random.default_rng(3)
    n = 1 << 16
    rays = np.zeros(n, capi.RAY_DTYPE)
    rays["org"] = rng.uniform(0.05, 0.95, (n, 3))
    d = rng.normal(size=(n, 3))
    rays["dir"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays["tmax"] = 1e30
    with _api().Accel(sd) as acc:
        h = acc.trace_closest(rays)
    o = oracle.OracleScene(sd, use_bvh=True).trace_closest(rays)
    assert np.array_equal(h["prim"], o["prim"])
    hit = o["prim"] != capi.PB2_INVALID_PRIM
    assert np.array_equal(h["t"][hit].view(np.uint32), o["t"][hit].view(np.uint32))
    assert ((o["prim"] >= 10) & (o["prim"] < 34)).sum() > 1000  # the two instanced cubes
