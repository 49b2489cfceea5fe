"""Multi-GPU sharding of the render and traversal workloads.

The path has no data exchange: pixels x sample indices of a frame are independent, and so are the rays
of a batch.  Each rank (one process per GPU, ``torch.distributed``) renders its own contiguous range of
sample indices of every pixel; the frame is the sum of the ranks' RGBW films -- one all-reduce at the
end of a frame (NCCL on GPUs; gloo in the CPU tests).  Rays are split into contiguous chunks.
"""
from __future__ import annotations


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


def reduce_film(film, group=None):
    """Sums the ranks' RGBW films in place (torch tensor, any device)."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(film, op=dist.ReduceOp.SUM, group=group)
    return film


def render_sharded(pipeline, film, rank: int, world: int, group=None):
    """Renders this rank's sample range of the full frame into `film` and all-reduces it."""
    begin, count = sample_range(pipeline.settings.samples_per_pixel, rank, world)
    if count:
        pipeline.launch(film, None, begin, count)
    return reduce_film(film, group)
