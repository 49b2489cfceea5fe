"""The seeded scene generators: the tessellated Cornell-box variant covers exactly the room of the Cornell box
(same quads, same winding, the requested triangle count), and the batching workload draws variants of both the
Cornell-box and the mixed-materials generators with the configuration's ranges."""
import numpy as np

from piper2_b200 import scenes


def _tri_area_normal(v, ix):
    a, b, c = v[ix[:, 0]].astype(np.float64), v[ix[:, 1]].astype(np.float64), v[ix[:, 2]].astype(np.float64)
    return np.cross(b - a, c - a) * 0.5


def test_cornell_variant_tessellates_the_room():
    base = scenes.cornell_box(seed=5)
    var = scenes.cornell_variant(seed=5, triangles=40_000)
    assert 0.9 * 40_000 <= var.triangle_count <= 40_000
    for m0, m1 in zip(base.meshes, var.meshes):
        s0 = _tri_area_normal(m0.vertices, m0.indices).sum(axis=0)
        s1 = _tri_area_normal(m1.vertices, m1.indices).sum(axis=0)
        assert np.allclose(s0, s1, atol=1e-6)  # same area and orientation
        assert m0.material == m1.material
        lo0, hi0 = m0.vertices.min(axis=0), m0.vertices.max(axis=0)
        assert np.allclose(m1.vertices.min(axis=0), lo0) and np.allclose(m1.vertices.max(axis=0), hi0)
    assert bytes(var.settings.camera) == bytes(base.settings.camera)


def test_batch_workload_ranges():
    sds = scenes.batch_workload(seed=0)
    assert len(sds) == 64
    kinds = [sd.name.split()[1] for sd in sds]
    assert 16 <= kinds.count("cornell") <= 48 and kinds.count("mixed") == 64 - kinds.count("cornell")
    for sd in sds:
        st = sd.settings
        assert 128 <= st.width <= 1024 and st.samples_per_pixel in (4, 8, 16, 32, 64)
        assert 5_000 <= sd.triangle_count <= 2_100_000
