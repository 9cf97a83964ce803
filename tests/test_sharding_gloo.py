"""Multi-rank sharding of the texel path, on CPU ranks over gloo (world size 2).

Each rank traces its contiguous range of surface texels with the CPU oracle
(the same per-unit computation the GPU kernels reproduce bit for bit), the
ranks all-gather their payload slots, and the gathered result must equal the
single-process run over every texel exactly. This checks the partition
(every unit once, no overlap) and that a unit's result does not depend on
which rank or range computed it.
"""

import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _scene():
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout

    node = scenes.terrain_boxes(seed=2, grid=33, boxes=12)
    layout = MeshColorsLayout.build(node, texels_per_unit=4.0, min_resolution=2, max_resolution=8)
    return node, layout


def _trace(node, layout, units):
    from oracle.oracle import OracleScene

    orc = OracleScene(**node.pack())
    slots = np.zeros((layout.total_payload_count, 4), np.uint32)
    for it in range(2):
        orc.trace_texels(node.lighting, slots, layout.face_array, layout.instance_array, layout.side_array, units,
                         it, 1, 3, it == 0, threads=1)
    return slots


def _worker(rank, world, port, out_path):
    import sys

    sys.path.insert(0, str(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    import torch
    import torch.distributed as dist

    from nan_b200.parallel import payload_slots_of_texels, shard_range

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    node, layout = _scene()
    begin, end = shard_range(layout.total_surface_texels, rank, world)
    slots = _trace(node, layout, layout.units()[begin:end])
    mine = payload_slots_of_texels(layout, begin, end)
    mask = np.zeros(layout.total_payload_count, np.int32)
    mask[mine] = 1
    t_slots = torch.from_numpy(slots.view(np.int32).copy())
    t_mask = torch.from_numpy(mask)
    gathered = [torch.zeros_like(t_slots) for _ in range(world)]
    masks = [torch.zeros_like(t_mask) for _ in range(world)]
    dist.all_gather(gathered, t_slots)
    dist.all_gather(masks, t_mask)
    if rank == 0:
        merged = np.zeros_like(slots)
        owners = np.zeros(layout.total_payload_count, np.int32)
        for g, m in zip(gathered, masks):
            m = m.numpy().astype(bool)
            merged[m] = g.numpy().view(np.uint32)[m]
            owners += m
        np.savez(out_path, merged=merged, owners=owners)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_texel_shards_equal_single_run(tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "gathered.npz")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    data = np.load(out)
    node, layout = _scene()
    single = _trace(node, layout, layout.units())
    assert np.all(data["owners"] == 1)  # every payload slot written by exactly one rank
    np.testing.assert_array_equal(data["merged"], single)
    assert np.all(single[:, 3] == 2)


def test_shard_ranges_partition_units():
    from nan_b200.parallel import shard_range

    for total in (0, 1, 7, 1000, 12_635_868):
        for world in (1, 2, 3, 8):
            ranges = [shard_range(total, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)
