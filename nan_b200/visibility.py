"""PMR visibility SH on the GPU: the reference's visibility caster over this
package's BVH.

The reference bakes per-sample visibility as 16 spherical-harmonic
coefficients with a CPU caster (``trace_pmr_visibility_sh_tinybvh``,
vertex_baker/vertex_baking_utils.py:420-500, native code in
vertex_baker/cpp/tinybvh_visibility.cpp:145-230) and a hardware-ray-tracing
twin (``HWRTPMRVisibilitySHSampler``, vertex_baker/hwrt_visibility_baker.py:
145-240). This module keeps that sampler's name pattern, arguments and
defaults (512 rays, 0.5 ray length, 0.001 self bias) and runs the rays on the
GPU through ``nan_visibility_sh16``: the same direction table, origins and
summation order as the caster, so the SH output equals the caster's wherever
the two agree on which rays are blocked.
"""

from __future__ import annotations

import numpy as np

from ._native import check, lib, ptr, stream_handle

PMR_DEFAULT_RAY_COUNT = 512
PMR_DEFAULT_RAY_LENGTH = 0.5
PMR_DEFAULT_SELF_BIAS = 0.001
MAX_RAYS = 1024


def visibility_ray_table(ray_count: int = PMR_DEFAULT_RAY_COUNT) -> np.ndarray:
    """The caster's rays as f32[R, 20]: direction xyz, 0, 16 weighted SH values."""
    ray_count = int(ray_count)
    if not 1 <= ray_count <= MAX_RAYS:
        raise ValueError(f"ray_count must be in 1..{MAX_RAYS}, got {ray_count}")
    table = np.zeros((ray_count, 20), dtype=np.float32)
    check(lib().nan_visibility_ray_table(ray_count, table.ctypes.data))
    return table


def _as_device_f32x3(values, device, name: str):
    import torch

    t = torch.as_tensor(values, dtype=torch.float32)
    if t.ndim != 2 or t.shape[1] != 3:
        raise ValueError(f"{name} must have shape (N, 3), got {tuple(t.shape)}")
    return t.to(device).contiguous()


def trace_pmr_visibility_sh(scene, sample_positions, sample_normals, *, ray_count: int = PMR_DEFAULT_RAY_COUNT,
                            max_distance: float = PMR_DEFAULT_RAY_LENGTH, self_bias: float = PMR_DEFAULT_SELF_BIAS,
                            stream=None, table=None):
    """Visibility SH of every sample: (sh f32[S, 16], visible_counts i32[S]),
    both torch tensors on the scene's device. ``table`` (the result of
    ``visibility_ray_table`` already on the device) skips the table upload."""
    import torch

    device = scene.device.torch_device
    positions = _as_device_f32x3(sample_positions, device, "sample_positions")
    normals = _as_device_f32x3(sample_normals, device, "sample_normals")
    if normals.shape[0] != positions.shape[0]:
        raise ValueError("sample_positions and sample_normals must have matching lengths")
    if positions.shape[0] == 0:
        raise ValueError("at least one visibility sample is required")
    ray_count = int(ray_count)
    if table is None:
        table = torch.from_numpy(visibility_ray_table(ray_count)).to(device)
    elif tuple(table.shape) != (ray_count, 20):
        raise ValueError(f"table must have shape ({ray_count}, 20)")
    n = positions.shape[0]
    sh = torch.empty((n, 16), dtype=torch.float32, device=device)
    counts = torch.empty((n,), dtype=torch.int32, device=device)
    check(lib().nan_visibility_sh16(scene.context.handle, ptr(positions), ptr(normals), n, ptr(table), ray_count,
                                    float(max_distance), float(self_bias), ptr(sh), ptr(counts),
                                    stream_handle(stream)))
    return sh, counts


class PMRVisibilitySHSampler:
    """GPU counterpart of HWRTPMRVisibilitySHSampler: ``sample`` returns the
    per-sample visibility SH f32[S, 16]; the unoccluded ray counts of the last
    call are kept in ``visible_counts``."""

    def __init__(self, device):
        self.device = device
        self._tables: dict = {}
        self.visible_counts = None

    def sample(self, scene, sample_positions, sample_normals, *, ray_count: int = PMR_DEFAULT_RAY_COUNT,
               max_distance: float = PMR_DEFAULT_RAY_LENGTH, self_bias: float = PMR_DEFAULT_SELF_BIAS, stream=None):
        import torch

        ray_count = max(1, int(ray_count))
        table = self._tables.get(ray_count)
        if table is None:
            table = torch.from_numpy(visibility_ray_table(ray_count)).to(scene.device.torch_device)
            self._tables[ray_count] = table
        sh, self.visible_counts = trace_pmr_visibility_sh(scene, sample_positions, sample_normals,
                                                          ray_count=ray_count, max_distance=max_distance,
                                                          self_bias=self_bias, stream=stream, table=table)
        return sh
