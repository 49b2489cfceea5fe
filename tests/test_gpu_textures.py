"""Textured materials on the GPU: the textured room (checkerboard and 8-bit image textures with Repeat and Mirror
wrap, texcoords past [0, 1], textured roughness remapped per point, a textured material on a mesh without
texcoords) renders every sample bit-exact against the CPU oracle, whose texture arithmetic is pinned against the
reference's own texture kernels on the CPU; the batched renderer carries the textures of each scene."""
import numpy as np
import pytest

from piper2_b200 import scenes

pytestmark = pytest.mark.gpu


def _api():
    from piper2_b200 import api

    return api


@pytest.mark.parametrize("seed,size,spp", [(0, 48, 8), (1, 64, 4)])
def test_textured_room_samples_bitexact(oracle, seed, size, spp):
    sd = scenes.textured_room(seed=seed, width=size, height=size, spp=spp)
    with _api().Pipeline(sd) as pl:
        film, samples = pl.render(samples=True)
    ofilm, osamples = oracle.OracleScene(sd, use_bvh=True).render(sd.settings)
    diff = np.any(samples.view(np.uint32) != osamples.view(np.uint32), axis=-1)
    assert not diff.any(), f"{diff.sum()} of {diff.size} samples differ"
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)


def test_textures_change_the_image():
    sd = scenes.textured_room(seed=0, width=32, height=32, spp=4)
    flat = scenes.textured_room(seed=0, width=32, height=32, spp=4)
    for m in flat.materials:
        m.texture[:] = [0, 0, 0, 0]
    with _api().Pipeline(sd) as pl:
        a, _ = pl.render()
    with _api().Pipeline(flat) as pl:
        b, _ = pl.render()
    assert np.abs(a[..., :3] - b[..., :3]).sum() > 0.05 * np.abs(b[..., :3]).sum()


def test_batch_carries_textures():
    sds = [scenes.textured_room(seed=2, width=40, height=32, spp=4), scenes.cornell_box(seed=1, width=24, height=24)]
    ref = []
    for sd in sds:
        with _api().Pipeline(sd) as pl:
            ref.append(pl.render()[0])
    with _api().Batch(sds) as b:
        b.render()
        for i, r in enumerate(ref):
            np.testing.assert_allclose(b.film(i), r, rtol=1e-5, atol=1e-6)
