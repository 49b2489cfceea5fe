"""Multi-rank logic on CPU with the gloo backend (world size 2): each rank renders its share of the sample
indices (through the product's render_sharded, with a CPU stand-in for the GPU pipeline that renders with
the oracle), the films are all-reduced, and the sum equals the single-rank render within accumulation
rounding; ray batches split and re-join exactly; scenes of a batch are assigned by longest processing
time; the guide's gradient hook averages over ranks; a rank that fails is reported, not hung."""
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


class _OraclePipeline:
    """CPU stand-in for api.Pipeline in the gloo tests: renders sample ranges with the oracle into a torch
    film (the GPU pipeline's launch contract: add the samples of [begin, begin + count) to `film`)."""

    def __init__(self, sd):
        import oracle_py

        self.settings = sd.settings
        self._sc = oracle_py.OracleScene(sd, use_bvh=False)

    def launch(self, film, rect, sample_begin, sample_count):
        import torch

        f, _ = self._sc.render(self.settings, rect=rect, sample_begin=sample_begin, sample_count=sample_count,
                               threads=1, samples=False)
        film += torch.from_numpy(f)


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
        # the product's own sharded render, with the CPU stand-in pipeline
        t2 = torch.zeros((sd.settings.height, sd.settings.width, 4), dtype=torch.float32)
        D.render_sharded(_OraclePipeline(sd), t2, rank, world)
        # the guide's gradient hook: every rank ends with the mean of the ranks' gradients
        grad = torch.full((33840,), float(rank + 1), dtype=torch.float32)
        D.gradient_allreduce()(grad)
        if rank == 0:
            np.save(os.path.join(out_dir, "film.npy"), t.numpy())
            np.save(os.path.join(out_dir, "film_sharded.npy"), t2.numpy())
        np.save(os.path.join(out_dir, f"grad{rank}.npy"), grad.numpy())
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
    np.testing.assert_allclose(np.load(tmp_path / "film_sharded.npy"), full, rtol=1e-5, atol=1e-6)
    for r in range(2):
        assert np.all(np.load(tmp_path / f"grad{r}.npy") == 1.5)


def test_longest_processing_time_assignment():
    """Every scene goes to exactly one rank, heaviest first to the least-loaded rank, deterministically; no
    rank's load exceeds the mean plus the largest single cost (the greedy bound)."""
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        for n in (0, 1, 5, 64):
            costs = np.exp(rng.uniform(0, 8, n))
            parts = distributed.assign_scenes(costs, world)
            assert len(parts) == world
            flat = sorted(i for p in parts for i in p)
            assert flat == list(range(n))
            loads = [sum(costs[i] for i in p) for p in parts]
            if n:
                assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
            assert parts == distributed.assign_scenes(list(costs), world)
    # the largest scenes land on different ranks first
    assert distributed.assign_scenes([10, 9, 1, 1], 2) == [[0, 3], [1, 2]]


def test_scene_cost_orders_scenes():
    from piper2_b200 import scenes

    small = scenes.cornell_box(seed=0, width=64, height=64, spp=4)
    more_spp = scenes.cornell_box(seed=0, width=64, height=64, spp=16)
    bigger = scenes.cornell_box(seed=0, width=128, height=128, spp=4)
    assert distributed.scene_cost(small) < distributed.scene_cost(more_spp)
    assert distributed.scene_cost(small) < distributed.scene_cost(bigger)
    tris = scenes.triangle_soup(4096, seed=0)
    tris.settings = small.settings
    assert distributed.scene_cost(tris) > distributed.scene_cost(small)


def test_failing_rank_is_reported(tmp_path):
    port = _free_port()
    with pytest.raises(Exception):
        mp.spawn(_worker, args=(2, port, str(tmp_path), 1), nprocs=2, join=True)
