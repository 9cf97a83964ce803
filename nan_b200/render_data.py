"""String-keyed cache of output buffers (render_data.py:32-120 of the reference).

Passes ask for their outputs by key; the cache returns the same tensor while
the requested shape and dtype stay the same and reallocates otherwise.
Tensors are torch CUDA tensors used as plain buffers.
"""

from __future__ import annotations


class RenderData:
    def __init__(self, device):
        self.device = device
        self._textures: dict = {}
        self._buffers: dict = {}

    def _torch_device(self):
        return self.device.torch_device if hasattr(self.device, "torch_device") else self.device

    def get_texture(self, key: str, *, width: int, height: int, channels: int = 4, dtype=None, **_):
        """RGBA32F-style texture as a [height, width, channels] tensor (zeroed on creation)."""
        import torch

        dtype = dtype or torch.float32
        shape = (int(height), int(width), int(channels))
        t = self._textures.get(key)
        if t is None or tuple(t.shape) != shape or t.dtype != dtype:
            t = torch.zeros(shape, dtype=dtype, device=self._torch_device())
            self._textures[key] = t
        return t

    def get_buffer(self, key: str, *, size: int | None = None, struct_size: int | None = None,
                   element_count: int | None = None, **_):
        """Byte buffer as a 1-D uint8 tensor of `size` or struct_size*element_count bytes."""
        import torch

        if size is None:
            if struct_size is None or element_count is None:
                raise ValueError("get_buffer needs size or struct_size and element_count")
            size = int(struct_size) * int(element_count)
        size = int(size)
        b = self._buffers.get(key)
        if b is None or b.numel() != size:
            b = torch.zeros((size,), dtype=torch.uint8, device=self._torch_device())
            self._buffers[key] = b
        return b

    def release_texture(self, key: str) -> None:
        self._textures.pop(key, None)

    def release_buffer(self, key: str) -> None:
        self._buffers.pop(key, None)

    def clear(self) -> None:
        self._textures.clear()
        self._buffers.clear()
