"""Sharding of the path's independent units (texels, probes, pixels) over ranks.

Units are independent given the replicated scene, so N ranks each take one
contiguous range and no collective is needed on the data path; results can be
gathered once at the end. The range of rank r of N over T units is
[T*r//N, T*(r+1)//N): every unit exactly once, ranges ordered by rank.
"""

from __future__ import annotations


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    total, rank, world = int(total), int(rank), int(world)
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return total * rank // world, total * (rank + 1) // world


def payload_slots_of_texels(layout, begin: int, end: int):
    """Payload slot indices written by surface texels [begin, end): the front
    slot of each texel and, for double-sided instances, its back slot."""
    import numpy as np

    units = layout.units()[begin:end]
    inst = layout.instance_array[units[:, 0]]
    side = layout.side_array[units[:, 0]]
    front = inst[:, 2].astype(np.int64) + units[:, 1]
    two = (side[:, 1] & 1) == 1
    back = side[two, 0].astype(np.int64) + units[two, 1]
    return np.concatenate([front, back])
