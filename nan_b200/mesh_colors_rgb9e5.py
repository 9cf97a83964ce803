"""RGB9E5 pack pass (mesh_colors_rgb9e5.py:4-29 of the reference)."""

from __future__ import annotations

from ._native import check, lib, ptr, stream_handle


class MeshColorsRGB9E5Packer:
    """Pack float3 Mesh Colors irradiance (16-byte slots) into one uint per texel."""

    def __init__(self, device):
        self.device = device

    def execute(self, command_encoder, source, destination, texel_count: int) -> None:
        texel_count = max(0, int(texel_count))
        if texel_count == 0:
            return
        if source.numel() * source.element_size() < 16 * texel_count:
            raise ValueError("source holds fewer than texel_count 16-byte slots")
        if destination.numel() * destination.element_size() < 4 * texel_count:
            raise ValueError("destination holds fewer than texel_count uints")
        check(lib().nan_pack_rgb9e5(self.device.context.handle, ptr(source), ptr(destination), texel_count,
                                    stream_handle(command_encoder)))
