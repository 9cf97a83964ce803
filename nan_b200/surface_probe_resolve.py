"""Surface-probe resolve pass (surface_probe_resolve.py:16-112 of the reference).

execute() draws the scene through the camera lit by the probe field: per
pixel one primary ray; at the hit, the hit instance's probes are gathered
from its point octree (up to 96 candidates weighted by distance, plane
distance and normal, times a Chebyshev visibility prior from the radial
depth moments), the 32 strongest kept, a 2R fallback merged when their
effective sample size is below min_gather_count, and the irradiance
reconstructed; shaded as emissive + real-time sun + albedo / pi * irradiance.
debug_view 1-7 show the gather count, support, density, reconstruction
confidence, self-hit rate and the vertex-lighting views.

Vertex lighting (the reference's SurfaceProbeVertexLighting, a separate
bake) is optional here: without it the vertex-lighting lookups report
"not built", as the reference does before its first build.
"""

from __future__ import annotations

import ctypes
import time

from ._native import NanProbeLayoutDesc, NanProbeResolveOptions, check, lib, ptr, stream_handle
from .surface_probe_fields import DIFFUSE_IRRADIANCE_RGB_FIELD


def _numel(t, width: int) -> int:
    return int(t.numel() * t.element_size()) // width


class SurfaceProbeResolve:
    def __init__(self, device, scene, layout, geometry, *, profile_sink: list | None = None):
        start = time.perf_counter()
        self.device = device
        self.scene = scene
        self.layout = layout
        self.geometry = geometry
        g = geometry
        self._desc = NanProbeLayoutDesc(
            probes=ptr(g.probes), probe_count=int(g.probe_count), node_count=_numel(g.nodes, 16), nodes=ptr(g.nodes),
            instances=ptr(g.instances), instance_count=int(g.instance_count),
            triangle_vertex_probe_count=_numel(g.triangle_vertex_probes, 16),
            triangle_vertex_probes=ptr(g.triangle_vertex_probes))
        if profile_sink is not None:
            profile_sink.append(("resolve_pipeline_create", time.perf_counter() - start))

    def execute(self, command_encoder, field, attachments, output, *, debug_view: int = 0, min_gather_count: int = 4,
                use_vertex_fallback: bool = False, vertex_lighting=None, vertex_lighting_rgbm=None,
                vertex_lighting_target=None, use_vertex_lighting: bool = False,
                use_radial_visibility: bool = True) -> None:
        if field.desc != DIFFUSE_IRRADIANCE_RGB_FIELD:
            raise ValueError("SurfaceProbeResolve currently consumes evaluated diffuse irradiance RGB")
        if output.dim() != 3 or output.shape[2] != 4 or not output.is_contiguous():
            raise ValueError("output must be a contiguous [H, W, 4] float32 tensor")
        h, w = int(output.shape[0]), int(output.shape[1])
        opt = NanProbeResolveOptions(
            debug_view=max(0, min(7, int(debug_view))), min_gather_count=max(1, min(32, int(min_gather_count))),
            use_vertex_fallback=int(bool(use_vertex_fallback)), use_vertex_lighting=int(bool(use_vertex_lighting)),
            use_radial_visibility=int(bool(use_radial_visibility)),
            frame_index=int(getattr(self.scene, "frame_index", 0)) & 0xFFFFFFFF,
            max_density_multiplier=float(self.layout.max_density_multiplier), vertex_lighting_rgbm_range=1.0)
        built = (vertex_lighting is not None and vertex_lighting_rgbm is not None and vertex_lighting_target is not None
                 and bool(getattr(vertex_lighting, "built", False)))
        if built:
            tri_map = vertex_lighting.triangle_map_buffer
            offsets = vertex_lighting.instance_offsets_buffer
            if _numel(offsets, 8) < int(self.geometry.instance_count):
                raise ValueError("vertex-lighting instance offsets must cover every probe-layout instance")
            opt.vertex_lighting_rgbm = ptr(vertex_lighting_rgbm)
            opt.vertex_lighting_target = ptr(vertex_lighting_target)
            opt.vertex_lighting_triangle_map = ptr(tri_map)
            opt.vertex_lighting_instance_offsets = ptr(offsets)
            opt.vertex_lighting_vertex_count = min(_numel(vertex_lighting_rgbm, 4), _numel(vertex_lighting_target, 16))
            opt.vertex_lighting_triangle_record_count = _numel(tri_map, 16)
            opt.vertex_lighting_rgbm_range = max(float(vertex_lighting.last_rgbm_range), 1.0)
        cam = self.scene.camera.to_struct()
        light = self.scene.lighting.to_struct()
        check(lib().nan_resolve_probes(self.scene.context.handle, ctypes.byref(self._desc), ptr(field.values),
                                       ptr(field.sample_counts), ptr(attachments.self_hit_counts),
                                       ptr(attachments.radial_moments), ctypes.byref(opt), ptr(output), w, h,
                                       ctypes.byref(cam), ctypes.byref(light), stream_handle(command_encoder)))
