"""Weighted sample elimination of surface-probe candidates on the GPU
(surface_probe_sampler.py / surface_probe_sampler.h:120-130 and
weighted_sample_elimination, surface_probes.py:1091-1123 of the reference).

SurfaceProbeSampler.eliminate thins many candidate sets in one call (one
persistent set of launches for all instances of a scene);
weighted_sample_elimination keeps the reference's single-set signature and
returns (selected indices ascending, Poisson radius). The elimination is the
reference's: largest weight first (lowest index on ties), weights
sum_j (1 - d_ij / d_max)^8 over compatible neighbours, run as parallel
rounds that remove every local maximum at once and give the same survivors.
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._native import Context, NanWseOptions, check, lib, ptr, stream_handle

WSE_NORMAL_COSINE_THRESHOLD = 0.5
WSE_PLANE_DISTANCE_SCALE = 0.35


class SurfaceProbeSampler:
    """Owns the context the elimination runs in."""

    def __init__(self, device):
        self.device = device
        index = getattr(device, "index", 0)
        self.context = Context(int(index))
        self.last_rounds = 0

    def eliminate(self, positions, normals, set_offsets, output_counts, surface_areas, *,
                  normal_cosine_threshold: float = WSE_NORMAL_COSINE_THRESHOLD,
                  plane_distance_scale: float = WSE_PLANE_DISTANCE_SCALE, stream=None):
        """positions, normals: float32 [N, 3] (CUDA tensors or arrays), the sets
        contiguous with boundaries set_offsets [S+1]. Returns (keep uint8 CUDA
        tensor [N], Poisson radius per set)."""
        import torch

        dev = self.device.torch_device if hasattr(self.device, "torch_device") else torch.device("cuda")
        pos = torch.as_tensor(positions, dtype=torch.float32, device=dev).reshape(-1, 3).contiguous()
        nrm = torch.as_tensor(normals, dtype=torch.float32, device=dev).reshape(-1, 3).contiguous()
        off = np.ascontiguousarray(set_offsets, dtype=np.uint32).reshape(-1)
        outs = np.ascontiguousarray(output_counts, dtype=np.uint32).reshape(-1)
        areas = np.ascontiguousarray(surface_areas, dtype=np.float32).reshape(-1)
        sets = off.shape[0] - 1
        if sets < 0 or outs.shape[0] != sets or areas.shape[0] != sets or int(off[-1]) != pos.shape[0]:
            raise ValueError("set_offsets, output_counts and surface_areas must describe the candidate sets")
        keep = torch.zeros(pos.shape[0], dtype=torch.uint8, device=dev)
        radii = np.zeros(max(sets, 1), np.float32)
        rounds = ctypes.c_uint32(0)
        opt = NanWseOptions(float(normal_cosine_threshold), float(plane_distance_scale))
        check(lib().nan_wse_eliminate(self.context.handle, ptr(pos), ptr(nrm), off.ctypes.data, sets,
                                      outs.ctypes.data, areas.ctypes.data, ctypes.byref(opt), ptr(keep),
                                      radii.ctypes.data, ctypes.byref(rounds), stream_handle(stream)))
        self.last_rounds = int(rounds.value)
        return keep, radii[:sets]


def weighted_sample_elimination(positions, normals, output_count: int, *, surface_area: float,
                                normal_cosine_threshold: float = WSE_NORMAL_COSINE_THRESHOLD,
                                plane_distance_scale: float = WSE_PLANE_DISTANCE_SCALE, device=None):
    """Single-set form: (selected candidate indices ascending, Poisson radius)."""
    from .scene import Device

    n = int(np.asarray(positions).reshape(-1, 3).shape[0]) if not hasattr(positions, "shape") else int(
        positions.shape[0])
    if n == 0:
        raise ValueError("weighted sample elimination needs at least one candidate")
    sampler = SurfaceProbeSampler(device if device is not None else Device(0))
    keep, radii = sampler.eliminate(positions, normals, [0, n], [max(1, min(int(output_count), n))],
                                    [float(surface_area)], normal_cosine_threshold=normal_cosine_threshold,
                                    plane_distance_scale=plane_distance_scale)
    return np.flatnonzero(keep.cpu().numpy()).astype(np.int64), float(radii[0])
