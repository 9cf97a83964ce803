"""Immutable GPU surface-probe geometry (surface_probe_resources.py:24-89 of the reference).

Record layouts: probe 48 B {position_radius f32x4, normal_side f32x4,
meta u32x4 = (primitive, bary.y bits, bary.z bits, flags | instance << 8)},
instance 48 B {root_center_extent f32x4, offsets u32x4, params f32x4 with
params.x = kernel radius}, octree node 16 B.
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

SURFACE_PROBE_METADATA_SIZE = 48
SURFACE_PROBE_NODE_SIZE = 16
SURFACE_PROBE_INSTANCE_SIZE = 48
SURFACE_PROBE_RADIAL_DEPTH_DIM = 4
SURFACE_PROBE_RADIAL_MOMENT_SIZE = SURFACE_PROBE_RADIAL_DEPTH_DIM * SURFACE_PROBE_RADIAL_DEPTH_DIM * 4
SURFACE_PROBE_FLAG_BACK_SIDE = 1 << 0
SURFACE_PROBE_FLAG_VERTEX_ANCHOR = 1 << 1
SURFACE_PROBE_FLAG_PROTECTED = 1 << 2
SURFACE_PROBE_INSTANCE_SHIFT = 8

SURFACE_PROBE_DTYPE = np.dtype(
    [("position_radius", np.float32, (4,)), ("normal_side", np.float32, (4,)), ("meta", np.uint32, (4,))],
    align=False)
SURFACE_PROBE_INSTANCE_DTYPE = np.dtype(
    [("root_center_extent", np.float32, (4,)), ("offsets", np.uint32, (4,)), ("params", np.float32, (4,))],
    align=False)


@dataclass(frozen=True)
class SurfaceProbeGpuGeometry:
    probes: object
    nodes: object
    instances: object
    triangle_vertex_probes: object
    probe_count: int
    instance_count: int

    @classmethod
    def create(cls, device, layout, *, profile_sink: list | None = None) -> "SurfaceProbeGpuGeometry":
        """Upload the layout's probe records, octree nodes, instance records and
        triangle->vertex-probe map. `device` is a nan_b200 Device (torch buffers)
        or any object with create_buffer(label=..., data=...)."""
        start = time.perf_counter()

        def mark(label):
            nonlocal start
            if profile_sink is not None:
                now = time.perf_counter()
                profile_sink.append((label, now - start))
                start = now

        def upload(label, data):
            if hasattr(device, "create_buffer"):
                return device.create_buffer(label=label, data=data)
            import torch
            raw = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
            return torch.from_numpy(raw.copy()).to(device.torch_device)

        probes = upload("surface_probe_metadata", np.ascontiguousarray(layout.probes).view(np.uint8))
        mark("gpu_probe_metadata_buffer")
        nodes = upload("surface_probe_nodes", np.ascontiguousarray(layout.nodes))
        mark("gpu_octree_buffer")
        instances = upload("surface_probe_instances", np.ascontiguousarray(layout.instance_gpu_data).view(np.uint8))
        mark("gpu_instance_buffer")
        tvp = upload("surface_probe_triangle_vertex_map", np.ascontiguousarray(layout.triangle_vertex_probes))
        mark("gpu_triangle_vertex_map_buffer")
        return cls(probes, nodes, instances, tvp, int(layout.total_probe_count), len(layout.instance_infos))
