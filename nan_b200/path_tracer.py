"""Screen path tracer pass (path_tracer.py:5-40 of the reference)."""

from __future__ import annotations

import ctypes

from ._native import check, lib, ptr, stream_handle


class PathTracer:
    """1 spp per frame unidirectional path tracer into an RGBA32F image.

    ``execute(command_encoder, output, frame)``: ``output`` is a float32
    CUDA tensor [H, W, 4]; ``command_encoder`` is a CUDA stream (or None for
    the current torch stream). ``max_vertices`` defaults to the reference's
    hard-coded 5 path vertices (path_tracer.slang:42).
    """

    def __init__(self, device, scene, *, max_vertices: int = 5):
        self.device = device
        self.scene = scene
        self.max_vertices = int(max_vertices)

    def execute(self, command_encoder, output, frame: int, static_shadow_mask=None,
                use_static_shadow_mask: bool = False) -> None:
        if use_static_shadow_mask and static_shadow_mask is not None:
            raise NotImplementedError("static shadow masks are not part of this path")
        if output.dim() != 3 or output.shape[2] != 4 or not output.is_contiguous():
            raise ValueError("output must be a contiguous [H, W, 4] float32 tensor")
        h, w = int(output.shape[0]), int(output.shape[1])
        self.scene.context.reserve_paths(w * h)  # wavefront scratch; grows only
        cam = self.scene.camera.to_struct()
        light = self.scene.lighting.to_struct()
        check(lib().nan_trace_screen(self.scene.context.handle, ptr(output), w, h, int(frame) & 0xFFFFFFFF,
                                     self.max_vertices, ctypes.byref(cam), ctypes.byref(light),
                                     stream_handle(command_encoder)))
