"""Surface-probe PRT L2 baker (surface_probe_prt.py:20-128 of the reference).

SurfaceProbePrtBaker.execute bakes, per probe, the transport of distant
light projected on the real orthonormal SH L2 basis (9 RGB coefficients) and
an RGB static source (emission and sun met along the paths), as running
means. SurfaceProbePrtEvaluator (surface_probe_prt.py:131-248) projects the
current escape radiance on the same basis and turns every probe's transport
into an irradiance field; evaluate_prt_l2_rgb is the same evaluation for one
probe on the host.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from ._native import check, lib, ptr, stream_handle
from .surface_probe_fields import DIFFUSE_IRRADIANCE_RGB_FIELD, DIFFUSE_PRT_L2_RGB_FIELD, SurfaceProbeRuntimeBuffers

SH_L2_CONSTANTS = (0.2820947918, 0.4886025119, 1.0925484306, 0.3153915653, 0.5462742153)


def surface_probe_sh_l2_basis(direction) -> np.ndarray:
    """The 9 basis values at a direction (float64)."""
    d = np.asarray(direction, dtype=np.float64)
    length = float(np.linalg.norm(d))
    if length <= 1e-12:
        raise ValueError("SH direction must be non-zero")
    x, y, z = d / length
    c0, c1, c2, c3, c4 = SH_L2_CONSTANTS
    return np.array([c0, c1 * y, c1 * z, c1 * x, c2 * x * y, c2 * y * z, c3 * (3.0 * y * y - 1.0), c2 * x * z,
                     c4 * (x * x - z * z)], dtype=np.float64)


def evaluate_prt_l2_rgb(transport, lighting_sh, static_source=(0.0, 0.0, 0.0)) -> np.ndarray:
    """max(static + sum_c transport[c] * lighting[c], 0), per channel."""
    t = np.asarray(transport, dtype=np.float64)
    l = np.asarray(lighting_sh, dtype=np.float64)
    if t.shape != (9, 3) or l.shape != (9, 3):
        raise ValueError("PRT transport and lighting SH must have shape (9, 3)")
    return np.maximum(np.asarray(static_source, dtype=np.float64) + np.sum(t * l, axis=0), 0.0)


def constant_environment_sh(radiance) -> np.ndarray:
    """SH L2 projection of a constant environment of the given radiance."""
    out = np.zeros((9, 3), np.float64)
    out[0] = np.asarray(radiance, dtype=np.float64) * np.sqrt(4.0 * np.pi)
    return out


class SurfaceProbePrtBaker:
    field_desc = DIFFUSE_PRT_L2_RGB_FIELD

    def __init__(self, device, scene, geometry, *, samples_per_probe: int = 1, max_bounces: int = 3,
                 profile_sink: list | None = None):
        start = time.perf_counter()
        self.device = device
        self.scene = scene
        self.geometry = geometry
        self.samples_per_probe = max(1, int(samples_per_probe))
        self.max_bounces = max(1, int(max_bounces))
        if profile_sink is not None:
            profile_sink.append(("prt_baker_pipeline_create", time.perf_counter() - start))

    def execute(self, command_encoder, field, attachments, iteration: int, *, reset: bool = False,
                probe_range: tuple[int, int] | None = None) -> None:
        if field.desc != self.field_desc:
            raise ValueError("SurfaceProbePrtBaker requires the L2 RGB PRT field")
        n = int(self.geometry.probe_count)
        begin, end = probe_range if probe_range is not None else (0, n)
        light = self.scene.lighting.to_struct()
        check(lib().nan_trace_probes_prt(
            self.scene.context.handle, ptr(field.values), ptr(field.sample_counts), ptr(attachments.self_hit_counts),
            ptr(attachments.radial_moments), ptr(attachments.static_source_rgb), ptr(self.geometry.probes), n,
            ptr(self.geometry.instances), int(self.geometry.instance_count), max(0, int(iteration)) & 0xFFFFFFFF,
            self.samples_per_probe, self.max_bounces, int(bool(reset)), ctypes.byref(light), int(begin), int(end),
            stream_handle(command_encoder)))


class SurfaceProbePrtEvaluator:
    LIGHTING_PROJECTION_SAMPLE_COUNT = 2048

    def __init__(self, device, scene, geometry, *, profile_sink: list | None = None):
        start = time.perf_counter()
        self.device = device
        self.scene = scene
        self.geometry = geometry
        if profile_sink is not None:
            profile_sink.append(("prt_evaluator_pipeline_create", time.perf_counter() - start))

    def lighting_signature(self) -> tuple[float, ...]:
        d = self.scene.lighting.sun_direction
        return float(d[0]), float(d[1]), float(d[2]), float(self.scene.lighting.sun_intensity)

    def acquire_evaluated_field(self, render_data):
        return SurfaceProbeRuntimeBuffers.acquire(render_data, self.geometry.probe_count,
                                                  field_desc=DIFFUSE_IRRADIANCE_RGB_FIELD, attachment_descs=(),
                                                  resource_prefix="surface_probe_renderer.prt_evaluated").field

    def execute(self, command_encoder, render_data, source_field, source_attachments, *,
                project_lighting: bool = True):
        if source_field.desc != DIFFUSE_PRT_L2_RGB_FIELD:
            raise ValueError("SurfaceProbePrtEvaluator requires the L2 RGB PRT field")
        lighting_sh = render_data.get_buffer("surface_probe_renderer.prt.lighting_sh", struct_size=16,
                                             element_count=9, label="surface_probe_prt_lighting_sh")
        evaluated = self.acquire_evaluated_field(render_data)
        stream = stream_handle(command_encoder)
        ctx = self.scene.context.handle
        if project_lighting:
            light = self.scene.lighting.to_struct()
            check(lib().nan_prt_project_lighting(ctx, ptr(lighting_sh), self.LIGHTING_PROJECTION_SAMPLE_COUNT,
                                                 ctypes.byref(light), stream))
        check(lib().nan_prt_evaluate(ctx, ptr(source_field.values), ptr(source_field.sample_counts),
                                     ptr(source_attachments.static_source_rgb), ptr(lighting_sh),
                                     ptr(evaluated.values), ptr(evaluated.sample_counts),
                                     int(self.geometry.probe_count), stream))
        return evaluated
