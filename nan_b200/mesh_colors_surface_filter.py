"""Mesh Colors one-ring surface filter (mesh_colors_surface_filter.py:12-130
of the reference): one pass of a normal-aware diffusion of the texel cache.
Each texel becomes the weighted mean of itself (weight 1) and its six
lattice neighbours (weight exp(-0.5 / spatial_sigma^2)). Neighbours across
a triangle edge are sampled in the adjacent face and also weighted by a
Gaussian in the angle between the face normals. All instances are filtered
in one launch.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from ._native import NanMeshColorsDesc, check, lib, ptr, stream_handle
from .mesh_colors import layout_adjacency, layout_face_normals


class MeshColorsSurfaceFilter:
    def __init__(self, device, scene, layout):
        import torch

        self.device = device
        self.scene = scene
        self.layout = layout
        dev = device.torch_device

        def up(a, dtype=torch.int32):
            return torch.from_numpy(np.ascontiguousarray(a).view(np.int32 if dtype == torch.int32 else np.float32)
                                    .copy()).to(dev)

        self._faces = up(layout.face_array)
        self._instances = up(layout.instance_array)
        self._sides = up(layout.side_array)
        self._prefix = up(layout.surface_prefix.astype(np.uint32))
        self.adjacency = up(layout_adjacency(scene.scene_node))
        self.face_normals = up(layout_face_normals(scene.scene_node), torch.float32)
        if self.adjacency.shape[0] != layout.face_array.shape[0]:
            raise ValueError("Mesh Colors adjacency count does not match the layout")
        d = NanMeshColorsDesc()
        d.face_infos = ptr(self._faces)
        d.face_count = layout.face_array.shape[0]
        d.instance_infos = ptr(self._instances)
        d.side_infos = ptr(self._sides)
        d.instance_count = layout.instance_array.shape[0]
        d.surface_prefix = ptr(self._prefix)
        d.total_surface_texels = layout.total_surface_texels
        d.payload_count = layout.total_payload_count
        self._desc = d

    def execute(self, command_encoder, source, destination, *, spatial_sigma: float = 1.0,
                normal_sigma_radians: float = math.radians(30.0)) -> None:
        if source.data_ptr() == destination.data_ptr():
            raise ValueError("Mesh Colors surface filtering requires ping-pong buffers")
        spatial_sigma = max(float(spatial_sigma), 1e-6)
        neighbor_weight = math.exp(-0.5 / (spatial_sigma * spatial_sigma))
        normal_sigma_radians = max(float(normal_sigma_radians), 0.0)
        check(lib().nan_filter_mesh_colors(self.scene.context.handle, ctypes.byref(self._desc), ptr(self.adjacency),
                                           ptr(self.face_normals), ptr(source), ptr(destination),
                                           ctypes.c_float(neighbor_weight), ctypes.c_float(normal_sigma_radians),
                                           stream_handle(command_encoder)))
