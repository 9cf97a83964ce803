"""Learned radiance cache: an online-trained irradiance cache over surface
points (no counterpart in the reference).

A multiresolution hash encoding (16 levels x 2 FP16 features x 2^log2_table
entries) of the position, plus the shading normal, feeds a 48-64-64-64-64-16
ReLU MLP whose first three outputs are irradiance RGB. The forward and
backward passes run in libnan_b200.so on the tensor cores (BF16 operands,
FP32 accumulation in TMEM); the loss is relative L2 and the optimizer Adam.

    cache = RadianceCache(device, bounds_min, bounds_max)
    cache.train(queries, targets, batch=16384)      # queries f32[N, 8], targets f32[N, 4]
    irradiance = cache.infer(queries)               # f32[N, 4]
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from ._native import NanCacheConfig, check, lib, ptr, stream_handle

LEVELS = 16
LAYER_SHAPES = ((64, 48), (64, 64), (64, 64), (64, 64), (16, 64))
MLP_PARAMS = sum(r * c for r, c in LAYER_SHAPES)
# hash-table optimizer step: Adam over every entry, or lazy Adam over the
# entries the step's samples touched
TABLE_UPDATES = {"dense": 0, "lazy": 1}


def initial_parameters(log2_table: int, seed: int = 0):
    """Glorot-uniform weights (output rows 3..15 zero) and a hash table
    uniform in [-1e-4, 1e-4]."""
    rng = np.random.default_rng(seed)
    ws = []
    for i, (r, c) in enumerate(LAYER_SHAPES):
        lim = math.sqrt(6.0 / ((r if i < 4 else 3) + c))
        w = rng.uniform(-lim, lim, size=(r, c)).astype(np.float32)
        if i == 4:
            w[3:, :] = 0.0
        ws.append(w)
    mlp = np.concatenate([w.reshape(-1) for w in ws]).astype(np.float32)
    table = rng.uniform(-1e-4, 1e-4, size=LEVELS * 2 * (1 << log2_table)).astype(np.float32)
    return mlp, table


def scene_bounds(scene, margin: float = 1e-3):
    """The scene's world-space box grown by `margin` x its largest extent on
    every side: the bounds a RadianceCache normalises positions to."""
    tris = scene.world_triangles().reshape(-1, 3)
    lo = tris.min(dim=0).values.cpu().numpy()
    hi = tris.max(dim=0).values.cpu().numpy()
    pad = margin * float((hi - lo).max())
    return tuple(float(x) - pad for x in lo), tuple(float(x) + pad for x in hi)


class RadianceCache:
    def __init__(self, device, bounds_min, bounds_max, *, log2_table: int = 19, base_resolution: int = 16,
                 max_resolution: int = 2048, learning_rate: float = 1e-2, beta1: float = 0.9, beta2: float = 0.99,
                 epsilon: float = 1e-15, loss_epsilon: float = 1e-2, table_update: str = "dense",
                 seed: int = 0):
        import torch

        self.device = device
        cfg = NanCacheConfig()
        for i in range(3):
            cfg.bounds_min[i] = float(bounds_min[i])
            cfg.bounds_max[i] = float(bounds_max[i])
        cfg.log2_table = int(log2_table)
        cfg.base_resolution = int(base_resolution)
        cfg.max_resolution = int(max_resolution)
        cfg.learning_rate = float(learning_rate)
        cfg.beta1 = float(beta1)
        cfg.beta2 = float(beta2)
        cfg.epsilon = float(epsilon)
        cfg.loss_epsilon = float(loss_epsilon)
        if table_update not in TABLE_UPDATES:
            raise ValueError(f"table_update must be one of {sorted(TABLE_UPDATES)}")
        cfg.table_update = TABLE_UPDATES[table_update]
        self.config = cfg
        n_mlp, n_table = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib().nan_cache_sizes(ctypes.byref(cfg), ctypes.byref(n_mlp), ctypes.byref(n_table)))
        self.mlp_params, self.table_params = int(n_mlp.value), int(n_table.value)
        self._context = device.new_context()
        handle = ctypes.c_void_p()
        check(lib().nan_cache_create(self._context.handle, ctypes.byref(cfg), ctypes.byref(handle)))
        self.handle = handle
        self._torch = torch
        mlp, table = initial_parameters(log2_table, seed)
        self.set_params(torch.from_numpy(mlp).to(device.torch_device), torch.from_numpy(table).to(device.torch_device))

    @property
    def context(self):
        return self._context

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            lib().nan_cache_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, mlp, table, stream=None) -> None:
        """Upload parameters (float32 device tensors) and reset Adam."""
        mlp = mlp.contiguous().float()
        table = table.contiguous().float()
        if mlp.numel() != self.mlp_params or table.numel() != self.table_params:
            raise ValueError("parameter sizes do not match the cache configuration")
        check(lib().nan_cache_set_params(self.handle, ptr(mlp), ptr(table), stream_handle(stream)))
        self._torch.cuda.current_stream().synchronize()

    def get_params(self, stream=None):
        t = self._torch
        mlp = t.empty(self.mlp_params, dtype=t.float32, device=self.device.torch_device)
        table = t.empty(self.table_params, dtype=t.float32, device=self.device.torch_device)
        check(lib().nan_cache_get_params(self.handle, ptr(mlp), ptr(table), None, None, None, stream_handle(stream)))
        return mlp, table

    def gradients(self, stream=None):
        """Accumulated MLP and table gradients and the accumulated loss."""
        t = self._torch
        g = t.empty(self.mlp_params, dtype=t.float32, device=self.device.torch_device)
        gt = t.empty(self.table_params, dtype=t.float32, device=self.device.torch_device)
        loss = t.empty(1, dtype=t.float32, device=self.device.torch_device)
        check(lib().nan_cache_get_params(self.handle, None, None, ptr(g), ptr(gt), ptr(loss), stream_handle(stream)))
        return g, gt, loss

    def infer(self, queries, out=None, stream=None):
        t = self._torch
        n = queries.shape[0]
        if out is None:
            out = t.empty((n, 4), dtype=t.float32, device=self.device.torch_device)
        check(lib().nan_cache_infer(self.handle, ptr(queries), n, ptr(out), stream_handle(stream)))
        return out

    def backward(self, queries, targets, batch: int | None = None, stream=None) -> None:
        n = queries.shape[0]
        check(lib().nan_cache_backward(self.handle, ptr(queries), ptr(targets), n, int(batch or n),
                                       stream_handle(stream)))

    def set_learning_rate(self, learning_rate: float) -> None:
        """Learning rate of the following optimizer steps."""
        check(lib().nan_cache_set_learning_rate(self.handle, float(learning_rate)))
        self.config.learning_rate = float(learning_rate)

    def step(self, stream=None) -> None:
        check(lib().nan_cache_step(self.handle, stream_handle(stream)))

    def train(self, queries, targets, batch: int = 16384, stream=None) -> None:
        check(lib().nan_cache_train(self.handle, ptr(queries), ptr(targets), queries.shape[0], int(batch),
                                    stream_handle(stream)))

    def check(self, stream=None) -> None:
        self._context.check(stream)
