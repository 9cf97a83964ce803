"""Oracle for the learned radiance cache (test infrastructure only).

CPU restatement, in numpy, of the cache that the CUDA kernels in
nan_b200/csrc/nan_cache.cu implement. It is the checker for the GPU's forward
values, gradients and optimizer updates; nothing in the product imports it.

The reference has no learned cache. The method restated here is published:
- multiresolution hash encoding: Mueller, Evans, Schied, Keller, "Instant
  Neural Graphics Primitives with a Multiresolution Hash Encoding" (2022),
  section 3 (per-level resolution N_l = floor(N_min * b**l); spatial hash
  x*1 ^ y*2654435761 ^ z*805459861 mod T; trilinear interpolation of the 8
  corners);
- online-trained radiance cache with a relative L2 loss: Mueller, Rousselle,
  Novak, Keller, "Real-time Neural Radiance Caching for Path Tracing" (2021),
  section 4;
- Adam: Kingma and Ba (2015), with bias correction.

Precision contract with the GPU:
- the encoding is evaluated in float32 in the kernel's operation order, so the
  32 hash features match the kernel bit for bit;
- every matrix product takes bf16-rounded operands (round to nearest even) and
  accumulates in float64 here (float32 in TMEM on the GPU);
- activations and back-propagated deltas are rounded to bf16 at the same
  points as in the kernel.
Agreement is therefore to float32 accumulation error, except where an fp32 vs
fp64 sum falls on the other side of a bf16 rounding boundary. The tests
state their tolerances.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

LEVELS = 16
FEATURES = 2
INPUTS = 48      # 32 hash features, normal xyz, constant 1, 12 zero pads
HIDDEN = 64
OUT_ROWS = 16    # output layer rows (3 used)
PRIMES = (1, 2654435761, 805459861)
LAYER_SHAPES = ((HIDDEN, INPUTS), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (OUT_ROWS, HIDDEN))
MLP_PARAMS = sum(r * c for r, c in LAYER_SHAPES)


@dataclass
class CacheConfig:
    log2_table: int = 19
    base_resolution: int = 16
    max_resolution: int = 2048
    bounds_min: tuple = (0.0, 0.0, 0.0)
    bounds_max: tuple = (1.0, 1.0, 1.0)
    lr: float = 1e-2
    beta1: float = 0.9
    beta2: float = 0.99
    eps: float = 1e-15
    loss_eps: float = 1e-2

    @property
    def table_size(self) -> int:
        return 1 << self.log2_table

    def resolutions(self) -> np.ndarray:
        b = math.exp((math.log(self.max_resolution) - math.log(self.base_resolution)) / (LEVELS - 1))
        return np.array([int(math.floor(self.base_resolution * b**l)) for l in range(LEVELS)], np.uint32)

    def inv_extent(self) -> np.ndarray:
        lo = np.asarray(self.bounds_min, np.float32)
        hi = np.asarray(self.bounds_max, np.float32)
        return (np.float32(1.0) / np.maximum(hi - lo, np.float32(1e-20))).astype(np.float32)


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (nearest even) and return as float32."""
    f = np.asarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def corner_lookup(cfg: CacheConfig, positions: np.ndarray):
    """Per level and corner: table index [n, L, 8] (uint32) and float32 weight.
    Follows the kernel's float32 operation order."""
    pos = np.asarray(positions, np.float32)
    lo = np.asarray(cfg.bounds_min, np.float32)
    p = (pos - lo) * cfg.inv_extent()
    p = np.clip(p, np.float32(0.0), np.float32(1.0))
    res = cfg.resolutions()
    T = cfg.table_size
    n = pos.shape[0]
    idx = np.zeros((n, LEVELS, 8), np.uint32)
    wts = np.zeros((n, LEVELS, 8), np.float32)
    for l in range(LEVELS):
        r = np.float32(res[l])
        s = p * r
        c = np.minimum(np.floor(s), r - np.float32(1.0))
        f = (s - c).astype(np.float32)
        ci = c.astype(np.uint64)
        one_m = (np.float32(1.0) - f).astype(np.float32)
        dense = (int(res[l]) + 1) ** 3 <= T
        stride = np.uint64(int(res[l]) + 1)
        for k in range(8):
            d = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1], np.uint64)
            g = ci + d
            if dense:
                ix = g[:, 0] + g[:, 1] * stride + g[:, 2] * stride * stride
            else:
                ix = ((g[:, 0] * np.uint64(PRIMES[0])) ^ (g[:, 1] * np.uint64(PRIMES[1])) ^
                      (g[:, 2] * np.uint64(PRIMES[2]))) & np.uint64(0xFFFFFFFF)
            idx[:, l, k] = (ix & np.uint64(T - 1)).astype(np.uint32)
            wx = np.where(d[0] == 1, f[:, 0], one_m[:, 0]).astype(np.float32)
            wy = np.where(d[1] == 1, f[:, 1], one_m[:, 1]).astype(np.float32)
            wz = np.where(d[2] == 1, f[:, 2], one_m[:, 2]).astype(np.float32)
            wts[:, l, k] = (wx * wy).astype(np.float32) * wz
    return idx, wts


def encode(cfg: CacheConfig, table_f16: np.ndarray, queries: np.ndarray) -> np.ndarray:
    """[n, 48] float32 network input: features in the kernel's summation order
    (corners 0..7, fp32), normal, constant 1, zero pads. queries: [n, 8]
    float32 (position xyz, pad, normal xyz, pad)."""
    q = np.asarray(queries, np.float32)
    tab = np.asarray(table_f16, np.float16).reshape(LEVELS, cfg.table_size, FEATURES).astype(np.float32)
    idx, wts = corner_lookup(cfg, q[:, 0:3])
    n = q.shape[0]
    x = np.zeros((n, INPUTS), np.float32)
    for l in range(LEVELS):
        a0 = np.zeros(n, np.float32)
        a1 = np.zeros(n, np.float32)
        for k in range(8):
            t = tab[l, idx[:, l, k]]
            a0 = (a0 + wts[:, l, k] * t[:, 0]).astype(np.float32)
            a1 = (a1 + wts[:, l, k] * t[:, 1]).astype(np.float32)
        x[:, 2 * l] = a0
        x[:, 2 * l + 1] = a1
    x[:, 32:35] = q[:, 4:7]
    x[:, 35] = 1.0
    return x


def split_weights(params: np.ndarray) -> list[np.ndarray]:
    out, off = [], 0
    for r, c in LAYER_SHAPES:
        out.append(np.asarray(params[off:off + r * c], np.float32).reshape(r, c))
        off += r * c
    return out


def forward(cfg, table_f16, params, queries, keep=False):
    """Network output [n, 3] (float64) and, with keep, the bf16 activations."""
    W = [bf16(w).astype(np.float64) for w in split_weights(params)]
    h = bf16(encode(cfg, table_f16, queries))
    acts = [h]
    a = h.astype(np.float64)
    for i in range(4):
        z = a @ W[i].T
        a = bf16(np.maximum(z, 0.0).astype(np.float32)).astype(np.float64)
        acts.append(a.astype(np.float32))
    out = a @ W[4].T
    if keep:
        return out[:, :3], acts, W
    return out[:, :3]


def loss_and_grads(cfg, table_f16, params, queries, targets, batch=None):
    """Relative L2 loss (mean over the batch of sum over channels of
    (o - y)^2 / (o^2 + eps), o held constant in the denominator) and its
    gradients: d/dparams [MLP_PARAMS] and d/dtable [L * T * 2], float64."""
    q = np.asarray(queries, np.float32)
    y = np.asarray(targets, np.float32)[:, :3].astype(np.float64)
    n = q.shape[0]
    B = float(batch if batch is not None else n)
    out, acts, W = forward(cfg, table_f16, params, q, keep=True)
    # the kernel reads o as float32 from TMEM
    o = out.astype(np.float32).astype(np.float64)
    denom = o * o + cfg.loss_eps
    loss = float(np.sum((o - y) ** 2 / denom) / B)
    d_out = np.zeros((n, OUT_ROWS), np.float64)
    d_out[:, :3] = 2.0 * (o - y) / (denom * B)
    delta = bf16(d_out.astype(np.float32)).astype(np.float64)
    grads = [None] * 5
    for i in range(4, -1, -1):
        a_in = acts[i].astype(np.float64)
        grads[i] = delta.T @ a_in
        g = delta @ W[i]
        if i > 0:
            delta = bf16(np.where(acts[i] > 0, g, 0.0).astype(np.float32)).astype(np.float64)
        else:
            g_in = g.astype(np.float32).astype(np.float64)  # read back as float32
    gp = np.concatenate([g.reshape(-1) for g in grads])
    # hash table gradient: scatter the input gradient of the 32 features
    idx, wts = corner_lookup(cfg, q[:, 0:3])
    gt = np.zeros((LEVELS, cfg.table_size, FEATURES), np.float64)
    for l in range(LEVELS):
        for k in range(8):
            w = wts[:, l, k].astype(np.float64)
            np.add.at(gt[l, :, 0], idx[:, l, k], w * g_in[:, 2 * l])
            np.add.at(gt[l, :, 1], idx[:, l, k], w * g_in[:, 2 * l + 1])
    return loss, gp, gt.reshape(-1)


def adam(cfg, param, m, v, grad, step, lazy=False):
    """One Adam step (float64); returns new (param, m, v). `step` counts from 1.

    lazy: the step applies only where the gradient is nonzero -- elsewhere the
    parameter and both moments stay as they are -- with the bias correction
    of the global step (lazy Adam, as for sparse embedding tables). The
    table's entries come in (feature 0, feature 1) pairs, and a pair is
    updated when either of its gradients is nonzero."""
    m1 = cfg.beta1 * m + (1.0 - cfg.beta1) * grad
    v1 = cfg.beta2 * v + (1.0 - cfg.beta2) * grad * grad
    mh = m1 / (1.0 - cfg.beta1**step)
    vh = v1 / (1.0 - cfg.beta2**step)
    p1 = param - cfg.lr * mh / (np.sqrt(vh) + cfg.eps)
    if not lazy:
        return p1, m1, v1
    g2 = grad.reshape(-1, 2)
    on = np.repeat((g2[:, 0] != 0) | (g2[:, 1] != 0), 2)
    return np.where(on, p1, param), np.where(on, m1, m), np.where(on, v1, v)


def init_params(cfg: CacheConfig, seed: int = 0):
    """Glorot-uniform MLP weights (output rows 3..15 zero) and a hash table
    uniform in [-1e-4, 1e-4] (as Instant NGP initialises it)."""
    rng = np.random.default_rng(seed)
    ws = []
    for i, (r, c) in enumerate(LAYER_SHAPES):
        lim = math.sqrt(6.0 / (r + c if i < 4 else 3 + c))
        w = rng.uniform(-lim, lim, size=(r, c)).astype(np.float32)
        if i == 4:
            w[3:, :] = 0.0
        ws.append(w)
    params = np.concatenate([w.reshape(-1) for w in ws]).astype(np.float32)
    table = rng.uniform(-1e-4, 1e-4, size=LEVELS * cfg.table_size * FEATURES).astype(np.float32)
    return params, table
