"""Multi-GPU sharding of trace jobs: one process per GPU, no collective on the data path.

Rays and scenes are independent, so a job splits into contiguous ranges of whole cameras (a batch of
scenes) or of image rows (one large frame), one range per rank. The only collectives are at the
end: a gather of the result arrays when one rank needs the whole frame, the sum of the adjoint's
scene-parameter gradients, and the maximum of the ranks' device times for reporting.
"""

from __future__ import annotations

from typing import Sequence


def shard_cameras(ray_counts: Sequence[int], world: int, rank: int) -> range:
    """Contiguous range of camera indices for `rank`, balancing rays across `world` ranks: rank k
    takes the cameras whose cumulative ray count starts in [k T / world, (k+1) T / world)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    total = sum(int(n) for n in ray_counts)
    lo = hi = None
    acc = 0
    for i, n in enumerate(ray_counts):
        owner = min(world - 1, (acc * world) // total) if total else 0
        if owner == rank:
            lo = i if lo is None else lo
            hi = i + 1
        acc += int(n)
    if lo is None:
        return range(0, 0)
    return range(lo, hi)


def shard_rows(height: int, world: int, rank: int) -> range:
    """Contiguous band of image rows for `rank` (the first height % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(int(height), world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def shard_region(width: int, height: int, world: int, rank: int):
    """The tile region of one frame that `rank` traces: a band of whole 8x8-pixel tile rows (the
    first ranks take one more row when the rows do not divide evenly), as a TileRegion for
    glc_camera.tile_origin / tile_count, or None when the rank has no rows. Its results land in the
    frame's own layout, so the ranks' bands together are the frame."""
    from .batches import TileRegion, tile_grid

    gx, gy = tile_grid(width, height)
    rows = shard_rows(gy, world, rank)
    if len(rows) == 0:
        return None
    return TileRegion((0, rows.start), (gx, len(rows)))


def region_pixel_rows(region, width: int, height: int) -> range:
    """Pixel rows a shard_region band covers (clipped to the frame)."""
    if region is None:
        return range(0, 0)
    _, y0, _, y1 = region.pixel_rect(width, height)
    return range(y0, y1)


def max_over_ranks(value: float, group=None) -> float:
    """The largest of the ranks' values (device times are reported as the slowest rank's)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_scene_gradients(grad, group=None):
    """Sum of the ranks' dL/d(a, Q, inclination, r_obs) for a scene whose rays are sharded."""
    import torch.distributed as dist

    dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad


def gather_rows(local, height: int, group=None):
    """Every rank's row band of a (rows, ...) array, concatenated in row order on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    parts = []
    for r in range(world):
        rows = shard_rows(height, world, r)
        parts.append(torch.empty((len(rows),) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device))
    # pad to the largest band so that all_gather sees equal shapes
    n = max(p.shape[0] for p in parts)
    pad = torch.zeros((n,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([b[: p.shape[0]] for b, p in zip(bufs, parts)], dim=0)
