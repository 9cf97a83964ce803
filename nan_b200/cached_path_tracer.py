"""Screen path tracer with a learned radiance cache (no counterpart in the
reference, whose PathTracer this extends: path_tracer.py:5-40).

Each frame traces the reference's path up to vertex `cache_vertex`:
- cache_vertex = 1 (default): up to the second hit; the rest of the path is
  throughput * albedo / pi * cache irradiance at that hit;
- cache_vertex = 0: the first hit with its sun NEE; the indirect light is
  albedo / pi * the cache's indirect irradiance at the first hit.

The cache trains online on the same frame. `train_samples` of the frame's
cache points, one per pixel in a per-frame strided set, get a plain estimate
of the cached quantity: the texel estimator with max_vertices - 1 -
cache_vertex hits, without its direct-sun term for cache_vertex = 0. They
are used for one pass of Adam steps in batches of `train_batch`. The targets
therefore have the expectation of the plain PathTracer's remaining path, so
the plain path tracer with `max_vertices` is the unbiased judge of the
cached frames.
"""

from __future__ import annotations

import ctypes
import math

from ._native import NanCachedFrame, check, lib, ptr, stream_handle


def _coprime_stride(p: int) -> int:
    """A stride near p * (golden ratio - 1) that is coprime with p."""
    if p <= 1:
        return 1
    s = max(1, int(p * 0.6180339887498949)) | 1
    while math.gcd(s, p) != 1:
        s += 2
    return s % p


class CachedPathTracer:
    def __init__(self, device, scene, cache, *, cache_vertex: int = 1, max_vertices: int = 5,
                 train_samples: int = 65536, train_batch: int = 65536, train: bool = True):
        import torch

        self.device = device
        self.scene = scene
        self.cache = cache
        if cache_vertex not in (0, 1) or max_vertices < cache_vertex + 2:
            raise ValueError("cache_vertex must be 0 or 1, with max_vertices >= cache_vertex + 2")
        self.cache_vertex = int(cache_vertex)
        self.train_samples = int(train_samples)
        self.train_bounces = int(max_vertices) - 1 - self.cache_vertex
        self.train_batch = int(train_batch)
        self.train = bool(train)
        self._torch = torch
        self._pixels = 0

    def _scratch(self, p: int) -> None:
        if p == self._pixels:
            return
        t, dev = self._torch, self.device.torch_device
        self.queries = t.empty((p, 8), dtype=t.float32, device=dev)
        self.weights = t.empty((p, 4), dtype=t.float32, device=dev)
        self.query_count = t.zeros(4, dtype=t.int32, device=dev)
        n = min(self.train_samples, p)
        self.train_points = t.empty((max(n, 1), 4), dtype=t.float32, device=dev)
        self.train_queries = t.empty((max(n, 1), 8), dtype=t.float32, device=dev)
        self.targets = t.empty((max(n, 1), 4), dtype=t.float32, device=dev)
        self._train_n = n
        self._stride = _coprime_stride(p)
        self._inverse = pow(self._stride, -1, p) if p > 1 else 0
        self._pixels = p

    def execute(self, command_encoder, output, frame: int) -> None:
        if output.dim() != 3 or output.shape[2] != 4 or not output.is_contiguous():
            raise ValueError("output must be a contiguous [H, W, 4] float32 tensor")
        h, w = int(output.shape[0]), int(output.shape[1])
        p = w * h
        self._scratch(p)
        ctx = self.scene.context
        ctx.reserve_paths(max(p, self._train_n))
        cam = self.scene.camera.to_struct()
        light = self.scene.lighting.to_struct()
        fd = NanCachedFrame()
        fd.queries = ptr(self.queries)
        fd.query_weights = ptr(self.weights)
        fd.query_count = ptr(self.query_count)
        fd.train_points = ptr(self.train_points)
        fd.train_queries = ptr(self.train_queries)
        fd.train_count = self._train_n if self.train else 0
        fd.train_offset = (int(frame) * 2654435761) % p
        fd.train_stride = self._stride
        fd.train_stride_inverse = self._inverse
        fd.cache_vertex = self.cache_vertex
        stream = stream_handle(command_encoder)
        check(lib().nan_trace_screen_cached(ctx.handle, self.cache.handle, ptr(output), w, h, int(frame) & 0xFFFFFFFF,
                                            ctypes.byref(cam), ctypes.byref(light), ctypes.byref(fd), stream))
        if self.train and self._train_n:
            check(lib().nan_trace_points(ctx.handle, ptr(self.train_points), self._train_n, ptr(self.targets),
                                         int(frame) & 0xFFFFFFFF, 1, self.train_bounces,
                                         1 if self.cache_vertex == 0 else 0, ctypes.byref(light), stream))
            check(lib().nan_cache_train(self.cache.handle, ptr(self.train_queries), ptr(self.targets), self._train_n,
                                        self.train_batch, stream))
