"""Multi-rank logic on CPU with the gloo backend (world size 2): each rank renders its share of the sample
indices with the oracle, the films are all-reduced, and the sum equals the single-rank render within
accumulation rounding; ray batches split and re-join exactly; a rank that fails is reported, not hung."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from piper2_b200 import distributed


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir, fail_rank):
    import sys

    import torch
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import datetime

    import oracle_py

    from piper2_b200 import distributed as D
    from piper2_b200 import scenes

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        sd = scenes.cornell_box(seed=4, width=24, height=24, spp=8)
        begin, count = D.sample_range(sd.settings.samples_per_pixel, rank, world)
        if rank == fail_rank:
            raise RuntimeError("injected failure on the host")
        film, _ = oracle_py.OracleScene(sd, use_bvh=False).render(sd.settings, sample_begin=begin, sample_count=count,
                                                                  threads=1)
        t = torch.from_numpy(film)
        D.reduce_film(t)
        if rank == 0:
            np.save(os.path.join(out_dir, "film.npy"), t.numpy())
    finally:
        dist.destroy_process_group()


def test_sample_and_ray_ranges_partition():
    for spp in (1, 7, 16, 64):
        for world in (1, 2, 3, 8):
            ranges = [distributed.sample_range(spp, r, world) for r in range(world)]
            assert sum(c for _, c in ranges) == spp
            assert ranges[0][0] == 0
            for (b0, c0), (b1, _) in zip(ranges, ranges[1:]):
                assert b0 + c0 == b1


def test_two_rank_film_reduce_equals_full_render(tmp_path, oracle):
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path), -1), nprocs=2, join=True)
    reduced = np.load(tmp_path / "film.npy")
    from piper2_b200 import scenes

    sd = scenes.cornell_box(seed=4, width=24, height=24, spp=8)
    full, _ = oracle.OracleScene(sd, use_bvh=False).render(sd.settings, threads=1)
    np.testing.assert_allclose(reduced, full, rtol=1e-5, atol=1e-6)


def test_failing_rank_is_reported(tmp_path):
    port = _free_port()
    with pytest.raises(Exception):
        mp.spawn(_worker, args=(2, port, str(tmp_path), 1), nprocs=2, join=True)
