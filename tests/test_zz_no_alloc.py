"""The allocation-free closest-hit entry point (pb2_trace_closest_nalloc), for callers whose device
memory is owned by their own allocator or who cannot take cudaMalloc's implicit synchronisation: its
scratch is a fixed static device array, so it must give the same hits as the allocating path
(pb2_accel_create + pb2_trace_closest), call after call, at its size limit and at zero sizes, leave the
device's free memory unchanged, and refuse inputs beyond its limit.

Kept in its own file, collected last, so that a failure here comes after every other test ran.
"""
import ctypes as C

import numpy as np
import pytest

from piper2_b200 import capi, scenes

pytestmark = pytest.mark.gpu

MAX_TRIANGLES = 16384


def _world_triangles(sd):
    mesh = sd.meshes[0]
    return np.ascontiguousarray(mesh.vertices[mesh.indices.reshape(-1)].reshape(-1, 9), dtype=np.float32)


def _nalloc(tris, n_tris, d_rays, n_rays, hits):
    import torch

    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return capi.lib().pb2_trace_closest_nalloc(C.c_void_p(tris.data_ptr() if tris is not None else 0), n_tris,
                                               C.c_void_p(d_rays.data_ptr()), n_rays, C.c_void_p(hits.data_ptr()),
                                               stream)


def _check_against_allocating_path(soup, rays, calls=2):
    import torch

    from piper2_b200 import api

    with api.Accel(soup) as acc:
        expected = acc.trace_closest(rays)
    tris = torch.from_numpy(_world_triangles(soup)).cuda()
    d_rays = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda()
    for call in range(calls):
        hits = torch.full((len(rays), 4), -1.0, dtype=torch.float32, device="cuda")
        capi.check(_nalloc(tris, tris.shape[0], d_rays, len(rays), hits))
        torch.cuda.synchronize()
        got = hits.cpu().numpy().copy().view(capi.HIT_DTYPE).reshape(-1)
        assert np.array_equal(got["prim"], expected["prim"]), f"call {call}: primitive ids differ"
        hit = expected["prim"] != capi.PB2_INVALID_PRIM
        for f in ("t", "u", "v"):
            assert np.array_equal(got[f][hit].view(np.uint32), expected[f][hit].view(np.uint32)), (call, f)
        assert hit.mean() > 0.05


def test_nalloc_matches_allocating_path_twice():
    _check_against_allocating_path(scenes.triangle_soup(12_000, seed=21),
                                   scenes.soup_rays(60_000, seed=22, kind="closest"))


def test_nalloc_at_its_triangle_limit():
    """Exactly MAX_TRIANGLES: the BVH, its build temporaries and CUB's sort space must still fit."""
    _check_against_allocating_path(scenes.triangle_soup(MAX_TRIANGLES, seed=23),
                                   scenes.soup_rays(20_000, seed=24, kind="closest"), calls=1)


def test_nalloc_zero_sizes():
    """No triangles: every ray misses.  No rays: nothing is written and the call succeeds."""
    import torch

    rays = scenes.soup_rays(1000, seed=25, kind="closest")
    d_rays = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda()
    hits = torch.zeros((len(rays), 4), dtype=torch.float32, device="cuda")
    capi.check(_nalloc(None, 0, d_rays, len(rays), hits))
    torch.cuda.synchronize()
    got = hits.cpu().numpy().copy().view(capi.HIT_DTYPE).reshape(-1)
    assert np.all(got["prim"] == capi.PB2_INVALID_PRIM)
    tris = torch.from_numpy(_world_triangles(scenes.triangle_soup(100, seed=26))).cuda()
    sentinel = torch.full((4, 4), 7.0, dtype=torch.float32, device="cuda")
    capi.check(_nalloc(tris, 100, d_rays, 0, sentinel))
    torch.cuda.synchronize()
    assert torch.all(sentinel == 7.0)


def test_nalloc_allocates_no_device_memory():
    """The point of the entry point: once its module is loaded (a first call), further calls leave the
    device's free memory exactly where it was (inputs and outputs are allocated before the reading)."""
    import torch

    soup = scenes.triangle_soup(8_000, seed=27)
    rays = scenes.soup_rays(30_000, seed=28, kind="closest")
    tris = torch.from_numpy(_world_triangles(soup)).cuda()
    d_rays = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda()
    hits = torch.zeros((len(rays), 4), dtype=torch.float32, device="cuda")
    capi.check(_nalloc(tris, tris.shape[0], d_rays, len(rays), hits))  # warm-up: lazy module loading
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        capi.check(_nalloc(tris, tris.shape[0], d_rays, len(rays), hits))
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, (free_before, free_after)


def test_nalloc_rejects_more_than_its_limit():
    import torch

    tris = torch.zeros((MAX_TRIANGLES + 1, 9), dtype=torch.float32, device="cuda")
    rays = torch.zeros((4, 8), dtype=torch.float32, device="cuda")
    hits = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    rc = capi.lib().pb2_trace_closest_nalloc(C.c_void_p(tris.data_ptr()), MAX_TRIANGLES + 1,
                                             C.c_void_p(rays.data_ptr()), 4, C.c_void_p(hits.data_ptr()), None)
    assert rc == 1
    assert b"16384" in capi.lib().pb2_last_error()
