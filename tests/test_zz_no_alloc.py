"""The allocation-free closest-hit entry point (pb2_trace_closest_nalloc), for callers whose device
memory is owned by their own allocator or who cannot take cudaMalloc's implicit synchronisation: its
scratch is a fixed static device array, so it must give the same hits as the allocating path
(pb2_accel_create + pb2_trace_closest), call after call, and refuse inputs beyond its limit.

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


def test_nalloc_matches_allocating_path_twice():
    import torch

    from piper2_b200 import api

    soup = scenes.triangle_soup(12_000, seed=21)
    rays = scenes.soup_rays(60_000, seed=22, kind="closest")
    with api.Accel(soup) as acc:
        expected = acc.trace_closest(rays)
    tris = torch.from_numpy(_world_triangles(soup)).cuda()
    d_rays = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        hits = torch.full((len(rays), 4), -1.0, dtype=torch.float32, device="cuda")
        capi.check(capi.lib().pb2_trace_closest_nalloc(C.c_void_p(tris.data_ptr()), tris.shape[0],
                                                       C.c_void_p(d_rays.data_ptr()), len(rays),
                                                       C.c_void_p(hits.data_ptr()), stream))
        torch.cuda.synchronize()
        got = hits.cpu().numpy().copy().view(capi.HIT_DTYPE).reshape(-1)
        assert np.array_equal(got["prim"], expected["prim"]), f"call {call}: primitive ids differ"
        hit = expected["prim"] != capi.PB2_INVALID_PRIM
        for f in ("t", "u", "v"):
            assert np.array_equal(got[f][hit].view(np.uint32), expected[f][hit].view(np.uint32)), (call, f)


def test_nalloc_rejects_more_than_its_limit():
    import torch

    tris = torch.zeros((MAX_TRIANGLES + 1, 9), dtype=torch.float32, device="cuda")
    rays = torch.zeros((4, 8), dtype=torch.float32, device="cuda")
    hits = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    rc = capi.lib().pb2_trace_closest_nalloc(C.c_void_p(tris.data_ptr()), MAX_TRIANGLES + 1,
                                             C.c_void_p(rays.data_ptr()), 4, C.c_void_p(hits.data_ptr()), None)
    assert rc == 1
    assert b"16384" in capi.lib().pb2_last_error()
