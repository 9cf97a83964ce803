"""Mesh Colors resolve pass (mesh_colors_resolve.py:8-73 of the reference).

execute() draws the accumulated texel cache (16-byte slots) seen through
the camera; execute_frozen() draws an RGB9E5-packed cache (the words of
MeshColorsRGB9E5Packer). One primary ray per pixel: the hit triangle's
lattice colours are interpolated and shaded as emissive + albedo / pi *
irradiance, misses show the sky.
"""

from __future__ import annotations

import ctypes

from ._native import check, lib, ptr, stream_handle


class MeshColorsResolve:
    def __init__(self, device, scene, layout, texture_space_path_tracer):
        self.device = device
        self.scene = scene
        self.layout = layout
        self.texture_space_path_tracer = texture_space_path_tracer

    def _run(self, command_encoder, mesh_colors, output, packed: bool) -> None:
        if output.dim() != 3 or output.shape[2] != 4 or not output.is_contiguous():
            raise ValueError("output must be a contiguous [H, W, 4] float32 tensor")
        h, w = int(output.shape[0]), int(output.shape[1])
        cam = self.scene.camera.to_struct()
        light = self.scene.lighting.to_struct()
        desc = self.texture_space_path_tracer._desc
        check(lib().nan_resolve_mesh_colors(self.scene.context.handle, ctypes.byref(desc), ptr(mesh_colors),
                                            int(packed), ptr(output), w, h, ctypes.byref(cam), ctypes.byref(light),
                                            stream_handle(command_encoder)))

    def execute(self, command_encoder, mesh_colors, output) -> None:
        self._run(command_encoder, mesh_colors, output, False)

    def execute_frozen(self, command_encoder, mesh_colors, output) -> None:
        self._run(command_encoder, mesh_colors, output, True)
