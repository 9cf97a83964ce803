"""Pinhole camera host state (camera.py:4-115 of the reference).

Computes the image-plane basis image_u/v/w and the Halton(2,3) sub-pixel
jitter that compute_ray_pinhole reads; everything in float32 like the
reference's spy.float3 math.
"""

from __future__ import annotations

import math

import numpy as np

from ._native import NanCamera


def halton(index: int, base: int) -> float:
    """Radical inverse of index in the given base (camera.py:4-11)."""
    result = 0.0
    factor = 1.0
    while index > 0:
        factor /= base
        result += factor * (index % base)
        index //= base
    return result


class HaltonSamplePattern:
    """Cycling Halton(2,3) pattern of sample_count points (camera.py:13-23)."""

    def __init__(self, sample_count: int):
        self.sample_count = sample_count
        self.current_sample = 0

    def next(self) -> np.ndarray:
        value = np.array([halton(self.current_sample, 2), halton(self.current_sample, 3)], dtype=np.float32)
        self.current_sample += 1
        if self.sample_count != 0:
            self.current_sample %= self.sample_count
        return value - np.floor(value)


def _normalize(v: np.ndarray) -> np.ndarray:
    v = np.asarray(v, dtype=np.float32)
    return (v / np.float32(np.sqrt(np.dot(v, v)))).astype(np.float32)


class Camera:
    def __init__(self):
        self.width = 100
        self.height = 100
        self.position = np.array([1, 1, 1], dtype=np.float32)
        self.target = np.array([0, 0, 0], dtype=np.float32)
        self.up = np.array([0, 1, 0], dtype=np.float32)
        self.fov = 70.0
        self.near_clip_plane = 0.03
        self.far_clip_plane = 1000.0
        self.focal_distance = 10000.0
        self.sample_pattern = HaltonSamplePattern(16)
        self.jitter = np.zeros(2, dtype=np.float32)
        self.frame_index = 0
        self.recompute()

    def recompute(self) -> None:
        """camera.py:45-80 (the raster matrices are not needed here)."""
        aspect = np.float32(self.width) / np.float32(self.height)
        fwd = _normalize(np.asarray(self.target, np.float32) - np.asarray(self.position, np.float32))
        self.image_w = (fwd * np.float32(self.focal_distance)).astype(np.float32)
        self.image_u = _normalize(np.cross(self.image_w, np.asarray(self.up, np.float32)).astype(np.float32))
        self.image_v = _normalize(np.cross(self.image_u, self.image_w).astype(np.float32))
        half = np.float32(math.tan(math.radians(self.fov) * 0.5))
        self.image_u = (self.image_u * (np.float32(self.focal_distance) * half * aspect)).astype(np.float32)
        self.image_v = (self.image_v * (np.float32(self.focal_distance) * half)).astype(np.float32)

    def begin_frame(self, w: int, h: int) -> None:
        """Advance the jitter pattern for a new frame (camera.py:87-96)."""
        self.width = w
        self.height = h
        sample = self.sample_pattern.next()
        self.jitter = (sample * np.array([1.0 / w, 1.0 / h], dtype=np.float32)).astype(np.float32)
        self.recompute()
        self.frame_index += 1

    def to_struct(self) -> NanCamera:
        c = NanCamera()
        c.position[:] = [float(x) for x in self.position]
        c.image_u[:] = [float(x) for x in self.image_u]
        c.image_v[:] = [float(x) for x in self.image_v]
        c.image_w[:] = [float(x) for x in self.image_w]
        c.jitter_x = float(self.jitter[0])
        c.jitter_y = float(self.jitter[1])
        c.near_clip = float(self.near_clip_plane)
        c.far_clip = float(self.far_clip_plane)
        return c
