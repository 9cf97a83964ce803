"""Progressive accumulation pass (accumulator.py:8-58 of the reference)."""

from __future__ import annotations

import time

from ._native import check, lib, ptr, stream_handle


class Accumulator:
    """RGBA32F running average: history += (rgb, 1); output = history.rgb / history.w."""

    def __init__(self, device, resource_key: str | None = None, *, profile_sink: list | None = None):
        start = time.perf_counter()
        self.device = device
        self.resource_key = resource_key or f"accumulator.history.{id(self)}"
        self.label = "accumulator"
        if profile_sink is not None:
            profile_sink.append(("accumulator_kernel_create", time.perf_counter() - start))

    def execute(self, command_encoder, render_data, input, output, reset: bool = False) -> None:
        h, w = int(input.shape[0]), int(input.shape[1])
        history = render_data.get_texture(self.resource_key, width=w, height=h)
        for t in (input, output, history):
            if tuple(t.shape) != (h, w, 4) or not t.is_contiguous():
                raise ValueError("accumulator textures must be contiguous [H, W, 4] float32 tensors")
        ctx = self.device.context.handle
        check(lib().nan_accumulate(ctx, ptr(input), ptr(output), ptr(history), w, h, int(bool(reset)),
                                   stream_handle(command_encoder)))
