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

    def _chunk_spans(self, begin: int, end: int, chunks: int):
        """Texel chunks of [begin, end) with the payload slot span each writes,
        or one whole-buffer chunk when a span is not contiguous (double-sided
        instances put back slots elsewhere)."""
        from .parallel import payload_slots_of_texels

        key = (begin, end, chunks)
        cached = getattr(self, "_spans", None)
        if cached is not None and cached[0] == key:
            return cached[1]
        spans = []
        for c in range(chunks):
            b = begin + (end - begin) * c // chunks
            e = begin + (end - begin) * (c + 1) // chunks
            if e <= b:
                continue
            slots = payload_slots_of_texels(self.layout, b, e)
            lo, hi = int(slots.min()), int(slots.max()) + 1
            if hi - lo != slots.shape[0]:
                spans = [(begin, end, 0, self.layout.total_payload_count)]
                break
            spans.append((b, e, lo, hi))
        self._spans = (key, spans)
        return spans

    def execute_host(self, host_slots, device_slots, iteration: int, *, reset: bool = False,
                     texel_range: tuple[int, int] | None = None, chunks: int = 2, stream=None) -> None:
        """One iteration on a payload held in pinned host memory: per texel
        chunk, the chunk's slots go host -> device on one copy stream, the
        chunk is traced on the compute stream and its slots come back on a
        second copy stream. A chunk's copies overlap the tracing of the other
        chunks, and of the previous and next iterations: the copy into chunk c
        waits only for chunk c's copy out of the previous call. The work is
        enqueued; ``host_ready(stream)`` makes a stream wait for the copies
        back. ``device_slots`` is the device staging buffer (payload size);
        ``host_slots`` must be pinned."""
        import torch

        if not host_slots.is_pinned():
            raise ValueError("host_slots must be in pinned memory")
        compute = stream if stream is not None else torch.cuda.current_stream()
        if getattr(self, "_copy_streams", None) is None:
            self._copy_streams = (torch.cuda.Stream(), torch.cuda.Stream())
            self._copied_out = None
        h2d, d2h = self._copy_streams
        begin, end = texel_range if texel_range is not None else (0, self.layout.total_surface_texels)
        spans = self._chunk_spans(int(begin), int(end), max(1, int(chunks)))
        host = host_slots.view(-1, 4) if host_slots.dim() != 2 else host_slots
        dev = device_slots.view(-1, 4) if device_slots.dim() != 2 else device_slots
        previous = self._copied_out
        if previous is None or len(previous) != len(spans):
            # first call, or other chunks: order after all earlier work
            h2d.wait_stream(compute)
            h2d.wait_stream(d2h)
            previous = [None] * len(spans)
        arrived = []
        for (b, e, lo, hi), out_event in zip(spans, previous):
            if out_event is not None:
                h2d.wait_event(out_event)
            with torch.cuda.stream(h2d):
                dev[lo:hi].copy_(host[lo:hi], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(h2d)
            arrived.append(ev)
        copied_out = []
        for (b, e, lo, hi), ev in zip(spans, arrived):
            compute.wait_event(ev)
            self.execute(compute, device_slots, iteration, reset=reset, texel_range=(b, e))
            done = torch.cuda.Event()
            done.record(compute)
            d2h.wait_event(done)
            with torch.cuda.stream(d2h):
                host[lo:hi].copy_(dev[lo:hi], non_blocking=True)
                out = torch.cuda.Event()
                out.record(d2h)
            copied_out.append(out)
        self._copied_out = copied_out

    def host_ready(self, stream=None) -> None:
        """Make `stream` (default: the current stream) wait until every slot
        copy of execute_host has reached the host buffer."""
        import torch

        streams = getattr(self, "_copy_streams", None)
        if streams is not None:
            (stream if stream is not None else torch.cuda.current_stream()).wait_stream(streams[1])
