"""Surface-probe diffuse irradiance baker (surface_probe_path_tracer.py:14-89 of the reference)."""

from __future__ import annotations

import ctypes
import time

from ._native import check, lib, ptr, stream_handle
from .surface_probe_fields import DIFFUSE_IRRADIANCE_RGB_FIELD


class SurfaceProbeDiffuseIrradianceBaker:
    """Per probe: samples_per_probe cosine samples in the face-normal frame,
    indirect light only, self-hit suspects, 4x4 hemi-oct radial depth
    moments (RG16F) and a running mean of the irradiance."""

    field_desc = DIFFUSE_IRRADIANCE_RGB_FIELD

    def __init__(self, device, scene, geometry, *, samples_per_probe: int = 1, max_bounces: int = 3,
                 profile_sink: list | None = None, compensated: bool = False):
        start = time.perf_counter()
        self.device = device
        self.scene = scene
        self.geometry = geometry
        self.samples_per_probe = max(1, int(samples_per_probe))
        self.max_bounces = max(1, int(max_bounces))
        scene.context.reserve_paths(max(1, int(geometry.probe_count)))  # wavefront scratch
        import torch

        # Kahan terms of the running means (compensated FP32); None keeps the
        # reference's plain lerp update
        self.compensation = (torch.zeros((max(1, int(geometry.probe_count)), 4), dtype=torch.float32,
                                          device=device.torch_device) if compensated else None)
        if profile_sink is not None:
            profile_sink.append(("trace_pipeline_create", time.perf_counter() - start))

    def execute(self, command_encoder, field, attachments, iteration: int, *, reset: bool = False,
                probe_range: tuple[int, int] | None = None) -> None:
        if field.desc != self.field_desc:
            raise ValueError("SurfaceProbeDiffuseIrradianceBaker requires the diffuse irradiance RGB field")
        n = int(self.geometry.probe_count)
        begin, end = probe_range if probe_range is not None else (0, n)
        light = self.scene.lighting.to_struct()
        check(lib().nan_trace_probes(
            self.scene.context.handle, ptr(field.values), ptr(field.sample_counts), ptr(attachments.self_hit_counts),
            ptr(attachments.radial_moments), ptr(self.geometry.probes), n, ptr(self.geometry.instances),
            int(self.geometry.instance_count), max(0, int(iteration)) & 0xFFFFFFFF, self.samples_per_probe,
            self.max_bounces, int(bool(reset)), ctypes.byref(light), int(begin), int(end),
            ptr(self.compensation), stream_handle(command_encoder)))


# Historical name kept by the reference for callers (surface_probe_path_tracer.py:86-89).
SurfaceProbePathTracer = SurfaceProbeDiffuseIrradianceBaker
