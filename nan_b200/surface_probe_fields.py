"""Surface-probe field descriptions and runtime buffers (surface_probe_fields.py of the reference)."""

from __future__ import annotations

from dataclasses import dataclass
from enum import Enum
from typing import Protocol

from .surface_probe_resources import SURFACE_PROBE_RADIAL_MOMENT_SIZE

SURFACE_PROBE_SAMPLE_COUNT_SIZE = 4
SURFACE_PROBE_SELF_HIT_SIZE = 4


class SurfaceProbeFieldSemantic(str, Enum):
    DIFFUSE_IRRADIANCE_RGB = "diffuse_irradiance_rgb"
    DIFFUSE_PRT_L2_RGB = "diffuse_prt_l2_rgb"


class SurfaceProbeFieldStorage(str, Enum):
    FLOAT32 = "float32"
    FLOAT16 = "float16"

    @property
    def scalar_size(self) -> int:
        return 4 if self is SurfaceProbeFieldStorage.FLOAT32 else 2


class SurfaceProbeAttachmentSemantic(str, Enum):
    SELF_HIT_COUNTS = "self_hit_counts"
    RADIAL_MOMENTS_4X4 = "radial_moments_4x4"
    STATIC_SOURCE_RGB = "static_source_rgb"


@dataclass(frozen=True)
class SurfaceProbeAttachmentDesc:
    semantic: SurfaceProbeAttachmentSemantic
    stride: int

    def __post_init__(self) -> None:
        if self.stride <= 0 or self.stride % 4 != 0:
            raise ValueError("Probe attachment stride must be positive and 4-byte aligned")


@dataclass(frozen=True)
class SurfaceProbeFieldDesc:
    semantic: SurfaceProbeFieldSemantic
    coefficient_count: int
    channel_count: int
    working_storage: SurfaceProbeFieldStorage
    version: int = 1

    def __post_init__(self) -> None:
        if self.coefficient_count <= 0:
            raise ValueError("Probe field coefficient count must be positive")
        if self.channel_count <= 0:
            raise ValueError("Probe field channel count must be positive")
        if self.version <= 0:
            raise ValueError("Probe field version must be positive")

    @property
    def value_stride(self) -> int:
        return self.coefficient_count * self.channel_count * self.working_storage.scalar_size

    @property
    def bytes_per_probe(self) -> int:
        return self.value_stride + SURFACE_PROBE_SAMPLE_COUNT_SIZE


DIFFUSE_IRRADIANCE_RGB_FIELD = SurfaceProbeFieldDesc(
    SurfaceProbeFieldSemantic.DIFFUSE_IRRADIANCE_RGB, 1, 3, SurfaceProbeFieldStorage.FLOAT32)
DIFFUSE_PRT_L2_RGB_FIELD = SurfaceProbeFieldDesc(
    SurfaceProbeFieldSemantic.DIFFUSE_PRT_L2_RGB, 9, 3, SurfaceProbeFieldStorage.FLOAT32)
SELF_HIT_COUNTS_ATTACHMENT = SurfaceProbeAttachmentDesc(
    SurfaceProbeAttachmentSemantic.SELF_HIT_COUNTS, SURFACE_PROBE_SELF_HIT_SIZE)
RADIAL_MOMENTS_4X4_ATTACHMENT = SurfaceProbeAttachmentDesc(
    SurfaceProbeAttachmentSemantic.RADIAL_MOMENTS_4X4, SURFACE_PROBE_RADIAL_MOMENT_SIZE)
STATIC_SOURCE_RGB_ATTACHMENT = SurfaceProbeAttachmentDesc(SurfaceProbeAttachmentSemantic.STATIC_SOURCE_RGB, 12)
DIFFUSE_IRRADIANCE_ATTACHMENTS = (SELF_HIT_COUNTS_ATTACHMENT, RADIAL_MOMENTS_4X4_ATTACHMENT)
DIFFUSE_PRT_ATTACHMENTS = (SELF_HIT_COUNTS_ATTACHMENT, RADIAL_MOMENTS_4X4_ATTACHMENT, STATIC_SOURCE_RGB_ATTACHMENT)


@dataclass(frozen=True)
class SurfaceProbeFieldBuffers:
    desc: SurfaceProbeFieldDesc
    values: object
    sample_counts: object


@dataclass(frozen=True)
class SurfaceProbeAttachments:
    buffers: dict

    def require(self, semantic: SurfaceProbeAttachmentSemantic):
        try:
            return self.buffers[semantic]
        except KeyError as error:
            raise ValueError(f"Surface Probe attachment is not available: {semantic.value}") from error

    @property
    def self_hit_counts(self):
        return self.require(SurfaceProbeAttachmentSemantic.SELF_HIT_COUNTS)

    @property
    def radial_moments(self):
        return self.require(SurfaceProbeAttachmentSemantic.RADIAL_MOMENTS_4X4)

    @property
    def static_source_rgb(self):
        return self.require(SurfaceProbeAttachmentSemantic.STATIC_SOURCE_RGB)


class SurfaceProbeFieldBaker(Protocol):
    field_desc: SurfaceProbeFieldDesc

    def execute(self, command_encoder, field: SurfaceProbeFieldBuffers, attachments: SurfaceProbeAttachments,
                iteration: int, *, reset: bool = False) -> None: ...


@dataclass(frozen=True)
class SurfaceProbeRuntimeBuffers:
    field: SurfaceProbeFieldBuffers
    attachments: SurfaceProbeAttachments

    @classmethod
    def acquire(cls, render_data, probe_count: int, *, field_desc: SurfaceProbeFieldDesc = DIFFUSE_IRRADIANCE_RGB_FIELD,
                attachment_descs: tuple = DIFFUSE_IRRADIANCE_ATTACHMENTS,
                resource_prefix: str = "surface_probe_renderer") -> "SurfaceProbeRuntimeBuffers":
        if field_desc.working_storage is not SurfaceProbeFieldStorage.FLOAT32:
            raise ValueError("Progressive Surface Probe fields currently require FP32")
        probe_count = max(1, int(probe_count))
        semantic = field_desc.semantic.value
        field_key = f"{resource_prefix}.field.{semantic}.v{field_desc.version}"
        values = render_data.get_buffer(f"{field_key}.values", size=field_desc.value_stride * probe_count,
                                        label=f"surface_probe_{semantic}_values")
        sample_counts = render_data.get_buffer(f"{field_key}.sample_counts", struct_size=SURFACE_PROBE_SAMPLE_COUNT_SIZE,
                                               element_count=probe_count, label="surface_probe_sample_counts")
        attachment_buffers = {}
        for desc in attachment_descs:
            if desc.semantic in attachment_buffers:
                raise ValueError(f"Duplicate Surface Probe attachment: {desc.semantic.value}")
            attachment_buffers[desc.semantic] = render_data.get_buffer(
                f"{field_key}.attachment.{desc.semantic.value}", struct_size=desc.stride, element_count=probe_count,
                label=f"surface_probe_{desc.semantic.value}")
        return cls(SurfaceProbeFieldBuffers(field_desc, values, sample_counts),
                   SurfaceProbeAttachments(attachment_buffers))
