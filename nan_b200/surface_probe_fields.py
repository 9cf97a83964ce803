"""Probe field descriptors and the per-probe buffers that a field bake writes.

A *field* is one running estimate per probe: ``value_stride`` bytes of
coefficients followed, in a separate buffer, by a 4-byte sample count.
*Attachments* are further per-probe records a baker keeps beside its field:
self-hit counts, radial depth moments, and the PRT bake's static source term.

Buffers are taken from a RenderData-style cache (``get_buffer(key, ...)``).
The keys follow ``"{prefix}.field.{semantic}.v{version}"`` and its
``.values``, ``.sample_counts`` and ``.attachment.{semantic}`` children, the
key scheme of the reference's field runtime (surface_probe_fields.py:185-236),
so a pass written against either finds the same resources. Names, semantic
strings and strides are the reference's drop-in interface
(surface_probe_fields.py:1-165); the code is this package's own.
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import Enum
from types import MappingProxyType
from typing import Mapping, Protocol

from .surface_probe_resources import SURFACE_PROBE_RADIAL_MOMENT_SIZE

SURFACE_PROBE_SAMPLE_COUNT_SIZE = 4
SURFACE_PROBE_SELF_HIT_SIZE = 4
_STATIC_SOURCE_RGB_SIZE = 12
_SCALAR_BYTES = {"float32": 4, "float16": 2}
_DEFAULT_PREFIX = "surface_probe_renderer"


class SurfaceProbeFieldSemantic(str, Enum):
    """What a field's coefficients mean."""

    DIFFUSE_IRRADIANCE_RGB = "diffuse_irradiance_rgb"
    DIFFUSE_PRT_L2_RGB = "diffuse_prt_l2_rgb"


class SurfaceProbeFieldStorage(str, Enum):
    """Scalar type of a field's coefficients."""

    FLOAT32 = "float32"
    FLOAT16 = "float16"

    @property
    def scalar_size(self) -> int:
        return _SCALAR_BYTES[self.value]


class SurfaceProbeAttachmentSemantic(str, Enum):
    """What an attachment's per-probe record holds."""

    SELF_HIT_COUNTS = "self_hit_counts"
    RADIAL_MOMENTS_4X4 = "radial_moments_4x4"
    STATIC_SOURCE_RGB = "static_source_rgb"


def _require_positive(owner: str, **values: int) -> None:
    for name, value in values.items():
        if int(value) <= 0:
            raise ValueError(f"{owner}: {name} must be a positive integer, got {value!r}")


@dataclass(frozen=True)
class SurfaceProbeAttachmentDesc:
    """An attachment: its semantic and the bytes of one probe's record."""

    semantic: SurfaceProbeAttachmentSemantic
    stride: int

    def __post_init__(self) -> None:
        _require_positive("probe attachment", stride=self.stride)
        if self.stride % 4:
            raise ValueError(f"probe attachment: stride {self.stride} is not a multiple of 4 bytes")


@dataclass(frozen=True)
class SurfaceProbeFieldDesc:
    """A field: coefficients x channels scalars of one storage type per probe."""

    semantic: SurfaceProbeFieldSemantic
    coefficient_count: int
    channel_count: int
    working_storage: SurfaceProbeFieldStorage
    version: int = 1

    def __post_init__(self) -> None:
        _require_positive("probe field", coefficient_count=self.coefficient_count,
                          channel_count=self.channel_count, version=self.version)

    @property
    def value_stride(self) -> int:
        """Bytes of one probe's coefficients."""
        return self.coefficient_count * self.channel_count * self.working_storage.scalar_size

    @property
    def bytes_per_probe(self) -> int:
        """Coefficients plus the sample count."""
        return self.value_stride + SURFACE_PROBE_SAMPLE_COUNT_SIZE

    def resource_key(self, prefix: str = _DEFAULT_PREFIX) -> str:
        """Cache key under which this field's buffers live."""
        return f"{prefix}.field.{self.semantic.value}.v{self.version}"


DIFFUSE_IRRADIANCE_RGB_FIELD = SurfaceProbeFieldDesc(
    SurfaceProbeFieldSemantic.DIFFUSE_IRRADIANCE_RGB, coefficient_count=1, channel_count=3,
    working_storage=SurfaceProbeFieldStorage.FLOAT32)
DIFFUSE_PRT_L2_RGB_FIELD = SurfaceProbeFieldDesc(
    SurfaceProbeFieldSemantic.DIFFUSE_PRT_L2_RGB, coefficient_count=9, channel_count=3,
    working_storage=SurfaceProbeFieldStorage.FLOAT32)

SELF_HIT_COUNTS_ATTACHMENT = SurfaceProbeAttachmentDesc(SurfaceProbeAttachmentSemantic.SELF_HIT_COUNTS,
                                                        SURFACE_PROBE_SELF_HIT_SIZE)
RADIAL_MOMENTS_4X4_ATTACHMENT = SurfaceProbeAttachmentDesc(SurfaceProbeAttachmentSemantic.RADIAL_MOMENTS_4X4,
                                                           SURFACE_PROBE_RADIAL_MOMENT_SIZE)
STATIC_SOURCE_RGB_ATTACHMENT = SurfaceProbeAttachmentDesc(SurfaceProbeAttachmentSemantic.STATIC_SOURCE_RGB,
                                                          _STATIC_SOURCE_RGB_SIZE)
DIFFUSE_IRRADIANCE_ATTACHMENTS = (SELF_HIT_COUNTS_ATTACHMENT, RADIAL_MOMENTS_4X4_ATTACHMENT)
DIFFUSE_PRT_ATTACHMENTS = DIFFUSE_IRRADIANCE_ATTACHMENTS + (STATIC_SOURCE_RGB_ATTACHMENT,)


@dataclass(frozen=True)
class SurfaceProbeFieldBuffers:
    """The buffers of one field: coefficients and per-probe sample counts."""

    desc: SurfaceProbeFieldDesc
    values: object
    sample_counts: object


class SurfaceProbeAttachments:
    """Read-only map from attachment semantic to its buffer.

    ``require`` (and the named properties) raise ``ValueError`` for an
    attachment that was not acquired, so a baker that needs one fails before
    it launches anything.
    """

    __slots__ = ("_by_semantic",)

    def __init__(self, buffers: Mapping) -> None:
        self._by_semantic = MappingProxyType(dict(buffers))

    @property
    def buffers(self) -> Mapping:
        return self._by_semantic

    def require(self, semantic: SurfaceProbeAttachmentSemantic):
        buffer = self._by_semantic.get(semantic)
        if buffer is None:
            raise ValueError(f"this field has no {SurfaceProbeAttachmentSemantic(semantic).value} attachment; "
                             "acquire it with the field's attachment_descs")
        return buffer

    @property
    def self_hit_counts(self):
        return self.require(SurfaceProbeAttachmentSemantic.SELF_HIT_COUNTS)

    @property
    def radial_moments(self):
        return self.require(SurfaceProbeAttachmentSemantic.RADIAL_MOMENTS_4X4)

    @property
    def static_source_rgb(self):
        return self.require(SurfaceProbeAttachmentSemantic.STATIC_SOURCE_RGB)

    def __repr__(self) -> str:
        return f"SurfaceProbeAttachments({sorted(s.value for s in self._by_semantic)})"


class SurfaceProbeFieldBaker(Protocol):
    """A pass that accumulates one field (and its attachments) per iteration."""

    field_desc: SurfaceProbeFieldDesc

    def execute(self, command_encoder, field: SurfaceProbeFieldBuffers, attachments: SurfaceProbeAttachments,
                iteration: int, *, reset: bool = False) -> None: ...


@dataclass(frozen=True)
class SurfaceProbeRuntimeBuffers:
    """A field's buffers and its attachments, taken from a buffer cache."""

    field: SurfaceProbeFieldBuffers
    attachments: SurfaceProbeAttachments

    @classmethod
    def acquire(cls, render_data, probe_count: int, *, field_desc: SurfaceProbeFieldDesc = DIFFUSE_IRRADIANCE_RGB_FIELD,
                attachment_descs: tuple = DIFFUSE_IRRADIANCE_ATTACHMENTS,
                resource_prefix: str = _DEFAULT_PREFIX) -> "SurfaceProbeRuntimeBuffers":
        """Get (or reuse) the buffers for ``probe_count`` probes.

        Progressive bakes keep float32 running means, so only float32 fields
        are accepted; each attachment semantic may appear once. A probe
        count below one still gets one probe's worth of storage.
        """
        if field_desc.working_storage is not SurfaceProbeFieldStorage.FLOAT32:
            raise ValueError(f"field {field_desc.semantic.value}: progressive bakes accumulate in float32, "
                             f"not {field_desc.working_storage.value}")
        seen = set()
        for desc in attachment_descs:
            if desc.semantic in seen:
                raise ValueError(f"attachment {desc.semantic.value} is listed twice")
            seen.add(desc.semantic)
        n = max(1, int(probe_count))
        key = field_desc.resource_key(resource_prefix)

        def buffer(suffix: str, **size):
            return render_data.get_buffer(f"{key}.{suffix}", label=f"{key}.{suffix}", **size)

        field = SurfaceProbeFieldBuffers(
            field_desc,
            values=buffer("values", size=field_desc.value_stride * n),
            sample_counts=buffer("sample_counts", struct_size=SURFACE_PROBE_SAMPLE_COUNT_SIZE, element_count=n))
        attachments = SurfaceProbeAttachments({
            desc.semantic: buffer(f"attachment.{desc.semantic.value}", struct_size=desc.stride, element_count=n)
            for desc in attachment_descs})
        return cls(field, attachments)
