"""Traversal parity on the GPU: closest-hit primitive ids and hit distances, and any-hit flags, through the
C ABI against the CPU oracle (same watertight test, brute force or BVH).  The bar is bit-exact: the
oracle and the CUDA kernels use the same triangle test operation for operation and the same
tie rule (lowest t, then lowest primitive id), so ids, t, u and v must be identical."""
import math

import numpy as np
import pytest

from piper2_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def _api():
    from piper2_b200 import api

    return api


def _assert_hits_equal(h, o):
    assert np.array_equal(h["prim"], o["prim"]), f"{np.count_nonzero(h['prim'] != o['prim'])} primitive ids differ"
    hit = o["prim"] != capi.PB2_INVALID_PRIM
    assert np.array_equal(h["t"][hit].view(np.uint32), o["t"][hit].view(np.uint32)), "hit distances differ"
    assert np.array_equal(h["u"][hit].view(np.uint32), o["u"][hit].view(np.uint32))
    assert np.array_equal(h["v"][hit].view(np.uint32), o["v"][hit].view(np.uint32))


@pytest.mark.parametrize("n_tris,n_rays", [(1, 64), (7, 512), (1000, 20000)])
def test_closest_and_any_vs_bruteforce(oracle, n_tris, n_rays):
    soup = scenes.triangle_soup(n_tris, seed=n_tris)
    for kind in ("closest", "any"):
        rays = scenes.soup_rays(n_rays, seed=n_tris + 7, kind=kind)
        o = oracle.OracleScene(soup, use_bvh=False)
        with _api().Accel(soup) as acc:
            if kind == "closest":
                _assert_hits_equal(acc.trace_closest(rays), o.trace_closest(rays))
            else:
                assert np.array_equal(acc.trace_any(rays), o.trace_any(rays))


def test_soup_medium_vs_bvh_oracle(oracle):
    soup = scenes.triangle_soup(200_000, seed=11)
    o = oracle.OracleScene(soup, use_bvh=True)
    with _api().Accel(soup) as acc:
        info = acc.info()
        assert info.triangle_count == 200_000 and info.node_count > 0
        rays = scenes.soup_rays(200_000, seed=12, kind="closest")
        _assert_hits_equal(acc.trace_closest(rays), o.trace_closest(rays))
        srays = scenes.soup_rays(200_000, seed=13, kind="any")
        assert np.array_equal(acc.trace_any(srays), o.trace_any(srays))


def test_full_size_stress_properties():
    """Traversal stress test at full size (1M triangles, 4M + 4M rays): hits must lie on the reported
    triangle (barycentric range), be inside (tmin, tmax), and a shadow ray cut at 0.999 t of a closest
    hit must be occluded iff the prefix contains another hit (checked against a closest-hit trace)."""
    soup = scenes.triangle_soup(1 << 20, seed=0)
    rays = scenes.soup_rays(1 << 22, seed=1, kind="closest")
    with _api().Accel(soup) as acc:
        h = acc.trace_closest(rays)
        hit = h["prim"] != capi.PB2_INVALID_PRIM
        assert hit.mean() > 0.5
        assert np.all(h["t"][hit] > rays["tmin"][hit]) and np.all(h["t"][hit] < rays["tmax"][hit])
        assert np.all(h["u"][hit] >= 0) and np.all(h["v"][hit] >= 0) and np.all(h["u"][hit] + h["v"][hit] <= 1.0001)
        # any-hit on [tmin, t_hit) never occludes when the closest hit is at t_hit (nothing nearer)
        cut = rays[hit][:500_000].copy()
        cut["tmax"] = h["t"][hit][:500_000]
        assert not acc.trace_any(cut).any()
        # ... and on (tmin, t_hit * 1.0001) it always does
        cut["tmax"] = h["t"][hit][:500_000] * np.float32(1.0001)
        assert acc.trace_any(cut).all()


def test_host_calls_chunked_equal_device_calls():
    """The host-array calls pipeline batches above 2^20 rays in chunks over three streams (2^20 rays each, a
    quarter and a half chunk at either end from 2^21 rays on); a 2.4M-ray batch (the ramped schedule, one body
    chunk partial) gives the same hits and flags as the device-pointer calls, and the same traversal counters."""
    import torch

    soup = scenes.triangle_soup(1 << 18, seed=4)
    n = (1 << 21) + 300_001
    rays = scenes.soup_rays(n, seed=5, kind="closest")
    srays = scenes.soup_rays(n, seed=6, kind="any")
    with _api().Accel(soup) as acc:
        acc.set_counting(True)
        h_host = acc.trace_closest(rays)
        c_host = acc.counters()
        o_host = acc.trace_any(srays)
        d_rays = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda()
        d_hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        acc.trace_closest_dev(d_rays.data_ptr(), n, d_hits.data_ptr())
        c_dev = acc.counters()
        d_srays = torch.from_numpy(srays.view(np.float32).reshape(-1, 8)).cuda()
        d_occ = torch.empty(n, dtype=torch.int32, device="cuda")
        acc.trace_any_dev(d_srays.data_ptr(), n, d_occ.data_ptr())
        torch.cuda.synchronize()
    h_dev = d_hits.cpu().numpy().view(capi.HIT_DTYPE).reshape(-1)
    assert np.array_equal(h_host.view(np.uint32), h_dev.view(np.uint32))
    assert np.array_equal(o_host, d_occ.cpu().numpy().view(np.uint32))
    assert c_host == c_dev and c_host[0] > n


def test_edge_cases(oracle):
    # shared edges and vertices (watertightness), degenerate triangles, rays along axes, empty batch
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0.5, 0.5, 0], [2, 2, 2], [2, 2, 2], [3, 3, 3]],
                 dtype=np.float32)
    ix = np.array([[0, 1, 2], [0, 2, 3], [0, 1, 4], [5, 6, 7], [4, 4, 4]], dtype=np.uint32)
    sd = scenes.SceneData(meshes=[scenes.MeshData(v, ix, 0)], materials=[scenes.material("Matte", (0.5, 0.5, 0.5))])
    g = np.linspace(0.0, 1.0, 33, dtype=np.float32)
    xs, ys = np.meshgrid(g, g)
    n = xs.size
    rays = np.zeros(n, dtype=capi.RAY_DTYPE)
    rays["org"][:, 0] = xs.ravel()
    rays["org"][:, 1] = ys.ravel()
    rays["org"][:, 2] = -1.0
    rays["dir"][:, 2] = 1.0
    rays["tmin"] = 0.0
    rays["tmax"] = 10.0
    o = oracle.OracleScene(sd, use_bvh=False)
    with _api().Accel(sd) as acc:
        _assert_hits_equal(acc.trace_closest(rays), o.trace_closest(rays))
        assert np.array_equal(acc.trace_any(rays), o.trace_any(rays))
        # every ray through the unit square hits (no cracks along the shared diagonal)
        inside = (rays["org"][:, 0] <= 1) & (rays["org"][:, 1] <= 1)
        assert np.all(acc.trace_closest(rays)["prim"][inside] != capi.PB2_INVALID_PRIM)
        # tmax == t of the hit: excluded (open interval)
        r2 = rays.copy()
        r2["tmax"] = 1.0
        assert not acc.trace_any(r2).any()
        # empty batch
        assert len(acc.trace_closest(rays[:0])) == 0


def test_empty_scene():
    sd = scenes.SceneData(materials=[scenes.material("Matte", (0.5, 0.5, 0.5))])
    with _api().Accel(sd) as acc:
        rays = scenes.soup_rays(100, seed=5)
        h = acc.trace_closest(rays)
        assert np.all(h["prim"] == capi.PB2_INVALID_PRIM)
        assert not acc.trace_any(rays).any()


def test_planes_and_cornell(oracle):
    sd = scenes.cornell_box(seed=3)
    rng = np.random.default_rng(0)
    n = 50_000
    rays = np.zeros(n, dtype=capi.RAY_DTYPE)
    rays["org"] = rng.uniform(0.05, 0.95, size=(n, 3))
    d = rng.normal(size=(n, 3))
    rays["dir"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays["tmin"] = 1e-3
    rays["tmax"] = 1e5
    o = oracle.OracleScene(sd, use_bvh=False)
    with _api().Accel(sd) as acc:
        h = acc.trace_closest(rays)
        _assert_hits_equal(h, o.trace_closest(rays))
        assert np.any(((h["prim"] & capi.PB2_PLANE_FLAG) != 0) & (h["prim"] != capi.PB2_INVALID_PRIM))
        assert np.array_equal(acc.trace_any(rays), o.trace_any(rays))


def test_counters_and_invalid_arguments():
    soup = scenes.triangle_soup(10_000, seed=1)
    with _api().Accel(soup) as acc:
        acc.set_counting(True)
        acc.trace_closest(scenes.soup_rays(1000, seed=2))
        nv, nt = acc.counters()
        assert nv >= 1000 and nt > 0
        with pytest.raises(capi.PB2Error):
            capi.check(capi.lib().pb2_trace_closest(acc.h, None, 10, None, None))


def _structure_scenes():
    return {
        "soup_1": scenes.triangle_soup(1, seed=2),
        "soup_9": scenes.triangle_soup(9, seed=2),
        "soup_100k": scenes.triangle_soup(100_000, seed=2),
        "cornell": scenes.cornell_box(seed=0),
        "guiding_room": scenes.guiding_room(seed=0, width=64, height=36),
    }


@pytest.mark.parametrize("name", ["soup_1", "soup_9", "soup_100k", "cornell", "guiding_room"])
def test_bvh_structure_validates(name):
    """Every child and triangle index in range and reached once; every triangle inside its child box."""
    sd = _structure_scenes()[name]
    with _api().Accel(sd) as acc:
        acc.validate()
        info = acc.info()
        assert info.triangle_count == sum(len(m.indices) for m in sd.meshes)


def test_guiding_room_traversal_vs_oracle(oracle):
    """Axis-aligned, coplanar, tessellated walls: closest and any hit against the oracle's BVH."""
    sd = scenes.guiding_room(seed=0, width=64, height=36)
    rng = np.random.default_rng(4)
    n = 100_000
    rays = np.zeros(n, dtype=capi.RAY_DTYPE)
    rays["org"] = rng.uniform((0.05, 0.05, 0.05), (3.95, 2.45, 3.95), size=(n, 3))
    d = rng.normal(size=(n, 3))
    d[: n // 10] = np.round(d[: n // 10])  # some axis-aligned and diagonal directions
    d[np.all(d == 0, axis=1)] = (0.0, 1.0, 0.0)
    rays["dir"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays["tmin"] = 1e-3
    rays["tmax"] = 1e5
    o = oracle.OracleScene(sd, use_bvh=True)
    with _api().Accel(sd) as acc:
        acc.validate()
        h = acc.trace_closest(rays)
        _assert_hits_equal(h, o.trace_closest(rays))
        assert np.array_equal(acc.trace_any(rays), o.trace_any(rays))
