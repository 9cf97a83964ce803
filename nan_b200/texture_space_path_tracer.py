"""Texture-space (Mesh Colors) tracer (texture_space_path_tracer.py:7-58 of the reference)."""

from __future__ import annotations

import ctypes

from ._native import NanMeshColorsDesc, check, lib, ptr, stream_handle


class TextureSpacePathTracer:
    """Per texel: one jittered lattice point, direct sun + a cosine path,
    running mean into the 16-byte slot (and the back slot when double sided).

    Unlike the reference, which issues one dispatch per instance
    (texture_space_path_tracer.py:42-58), all instances go in one launch.
    ``execute(command_encoder, output, iteration, reset=False)``: ``output``
    is the payload buffer (any CUDA tensor of payload_count * 16 bytes).
    ``texel_range`` restricts the launch to surface texels [begin, end).
    """

    def __init__(self, device, scene, layout, *, samples_per_texel: int = 1, max_bounces: int = 3,
                 max_paths_in_flight: int | None = None, compensated: bool = False):
        self.device = device
        self.scene = scene
        self.layout = layout
        self.samples_per_texel = max(1, int(samples_per_texel))
        self.max_bounces = max(1, int(max_bounces))
        (self.face_infos_buffer, self.instance_infos_buffer, self.side_infos_buffer,
         self.surface_prefix_buffer) = layout.create_gpu_buffers(device)
        d = NanMeshColorsDesc()
        d.face_infos = ptr(self.face_infos_buffer)
        d.face_count = layout.face_array.shape[0]
        d.instance_infos = ptr(self.instance_infos_buffer)
        d.side_infos = ptr(self.side_infos_buffer)
        d.instance_count = layout.instance_array.shape[0]
        d.surface_prefix = ptr(self.surface_prefix_buffer)
        d.total_surface_texels = layout.total_surface_texels
        d.payload_count = layout.total_payload_count
        # Kahan terms of the running means (compensated FP32); None keeps the
        # reference's plain lerp update
        import torch

        self.compensation = (torch.zeros((layout.total_payload_count, 4), dtype=torch.float32,
                                          device=device.torch_device) if compensated else None)
        d.compensation = ptr(self.compensation)
        self._desc = d
        # wavefront scratch: one path per surface texel in flight (or the cap)
        paths = layout.total_surface_texels if max_paths_in_flight is None else int(max_paths_in_flight)
        scene.context.reserve_paths(max(1, min(paths, layout.total_surface_texels)))

    def execute(self, command_encoder, output, iteration: int, *, reset: bool = False,
                texel_range: tuple[int, int] | None = None) -> None:
        if output.numel() * output.element_size() < 16 * self.layout.total_payload_count:
            raise ValueError("output holds fewer than total_payload_count 16-byte slots")
        begin, end = texel_range if texel_range is not None else (0, self.layout.total_surface_texels)
        light = self.scene.lighting.to_struct()
        check(lib().nan_trace_texels(self.scene.context.handle, ctypes.byref(self._desc), ptr(output),
                                     max(0, int(iteration)) & 0xFFFFFFFF, self.samples_per_texel, self.max_bounces,
                                     int(bool(reset)), ctypes.byref(light), int(begin), int(end),
                                     stream_handle(command_encoder)))
