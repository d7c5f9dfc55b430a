"""Batches of volumes over several GPUs: one process per GPU, no collective on the data path.

Volumes are independent units, so a batch is split across ranks by longest-first bin packing of
their estimated work (voxel counts): each volume goes to the rank with the least work so far,
largest volume first. Every rank skeletonizes its share with one `skeletonize_batch` call on its
own GPU; the only exchange is the final gather of the packed results to one rank (through
`torch.distributed.gather_object`, over whatever backend the process group has), where they are
put back in the batch's order.
"""
from __future__ import annotations

import heapq

import numpy as np

from . import batch as _batch


def partition(work, world):
    """Indices of the units per rank: longest first, each to the least-loaded rank (ties: lowest
    rank), each rank's list in ascending unit order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    heap = [(0, r) for r in range(world)]
    shares = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda i: (-int(work[i]), i)):
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + int(work[i]), r))
    return [sorted(s) for s in shares]


def iter_chunks(shape, chunk_shape, overlap=1):
    """Slices that tile a 3D `shape` with chunks of `chunk_shape` overlapping by `overlap` voxels
    (the reference's iter_chunks, src/brook/_pool.py:341-350): starts every chunk - overlap voxels
    along each axis, the last chunk clipped at the edge."""
    shape, chunk_shape = tuple(map(int, shape)), tuple(map(int, chunk_shape))
    if len(shape) != 3 or len(chunk_shape) != 3:
        raise ValueError("shape and chunk_shape must have three entries")
    starts = [range(0, max(s - overlap, 1), max(c - overlap, 1)) for s, c in zip(shape, chunk_shape)]
    for x in starts[0]:
        for y in starts[1]:
            for z in starts[2]:
                yield tuple(slice(a, min(a + c, s)) for a, c, s in zip((x, y, z), chunk_shape, shape))


def skeletonize_batch_sharded(samples, rank=None, world=None, dst=0, group=None, device=None, **options):
    """The batch `samples` (every rank passes the same list, or at least the same shapes) split over
    the ranks of the default process group; returns BatchedSkeletons for the whole batch on rank
    `dst` and None elsewhere. `options` are skeletonize_batch's (output is always packed)."""
    import torch.distributed as dist

    if rank is None:
        rank = dist.get_rank(group) if dist.is_initialized() else 0
    if world is None:
        world = dist.get_world_size(group) if dist.is_initialized() else 1
    options = dict(options)
    options.pop("output", None)
    anisotropy = options.get("anisotropy", (1, 1, 1))
    shares = partition([int(np.prod(np.shape(s))) for s in samples], world)
    mine = shares[rank]
    kwargs = dict(options, output="packed")
    if device is not None:
        kwargs["device"] = device
    result = _batch.skeletonize_batch([samples[i] for i in mine], **kwargs) if mine else None
    parts = {i: result[j] for j, i in enumerate(mine)} if result is not None else {}
    if world > 1:
        gathered = [None] * world if rank == dst else None
        dist.gather_object(parts, gathered, dst=dst, group=group)
        if rank != dst:
            return None
        for g in gathered:
            parts.update(g)
    from ._packed import PackedSkeletons

    ordered = [parts[i] if i in parts else PackedSkeletons.empty(anisotropy) for i in range(len(samples))]
    return _batch.BatchedSkeletons.concatenate(ordered, anisotropy)


__all__ = ["partition", "iter_chunks", "skeletonize_batch_sharded"]
