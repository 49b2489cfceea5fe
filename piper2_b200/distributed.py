"""Multi-GPU sharding of the render and traversal workloads.

The path has no data exchange: pixels x sample indices of a frame are independent, and so are the rays
of a batch and the scenes of a multi-scene batch.  One process per GPU (``torch.distributed``):

* a frame: each rank renders its own contiguous range of sample indices of every pixel, and the frame is
  the sum of the ranks' RGBW films -- one all-reduce at the end of the frame (NCCL on GPUs, gloo in the
  CPU tests);
* rays: contiguous chunks;
* many scenes (the batching workload): whole scenes go to ranks by greedy longest-processing-time on an
  estimated cost, no exchange; the films stay on the rank that rendered them unless gathered;
* guided rendering: the guiding network is trained on every rank from its own records, with the gradient
  of every training step averaged over the ranks (an all-reduce of 33,840 floats) so the ranks' networks
  stay identical.
"""
from __future__ import annotations

import math


def sample_range(spp: int, rank: int, world: int):
    """Contiguous share [begin, begin + count) of the sample indices 0..spp-1 for `rank`."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("invalid rank/world")
    base, extra = divmod(spp, world)
    begin = rank * base + min(rank, extra)
    count = base + (1 if rank < extra else 0)
    return begin, count


def ray_range(n: int, rank: int, world: int):
    return sample_range(n, rank, world)


def _world(group=None):
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(group)
    return 1


def reduce_film(film, group=None):
    """Sums the ranks' RGBW films in place (torch tensor, any device)."""
    import torch.distributed as dist

    if _world(group) > 1:
        dist.all_reduce(film, op=dist.ReduceOp.SUM, group=group)
    return film


def render_sharded(pipeline, film, rank: int, world: int, group=None):
    """Renders this rank's sample range of the full frame into `film` and all-reduces it.  `pipeline` is
    an :class:`piper2_b200.api.Pipeline` (or any object with ``settings.samples_per_pixel`` and
    ``launch(film, rect, sample_begin, sample_count)``)."""
    begin, count = sample_range(pipeline.settings.samples_per_pixel, rank, world)
    if count:
        pipeline.launch(film, None, begin, count)
    return reduce_film(film, group)


def scene_cost(scene_data) -> float:
    """Estimated render cost of one scene of a batch: its paths (film pixels x spp) times the traversal
    cost of a ray, which grows with the depth of its BVH (log2 of the triangle count), not with the count."""
    st = scene_data.settings
    tris = max(1, scene_data.triangle_count)
    return float(st.width) * float(st.height) * float(st.samples_per_pixel) * (1.0 + math.log2(tris))


def assign_scenes(costs, world: int):
    """Greedy longest-processing-time assignment of scenes to `world` ranks: scenes in decreasing cost (ties
    by index), each to the least-loaded rank (ties to the lowest rank).  Returns one sorted list of scene
    indices per rank; no rank carries more than the mean load plus the largest single cost."""
    if world <= 0:
        raise ValueError("world must be positive")
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += float(costs[i])
    return [sorted(x) for x in out]


def render_batch_sharded(scene_datas, rank: int, world: int, autotune: bool = True):
    """Renders this rank's share of a multi-scene batch (assign_scenes over scene_cost) in one batched launch
    on its GPU.  Returns {scene index: RGBW film (H x W x 4 numpy array)}; nothing is exchanged."""
    from . import api

    mine = assign_scenes([scene_cost(sd) for sd in scene_datas], world)[rank]
    if not mine:
        return {}
    with api.Batch([scene_datas[i] for i in mine]) as b:
        if autotune:
            b.autotune()
        b.render()
        return {i: b.film(k) for k, i in enumerate(mine)}


def gradient_allreduce(group=None):
    """A gradient hook (api.Guide.set_gradient_hook) that replaces each training step's gradient by its mean
    over the ranks of `group`, so every rank applies the same Adam update to the same network."""
    import torch.distributed as dist

    def hook(grad):
        world = _world(group)
        if world > 1:
            dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
            grad.div_(world)

    return hook
