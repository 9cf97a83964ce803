"""CPU restatement of the reference's PMR visibility caster, and a binding of
the caster itself. Test infrastructure: only tests/ and bench.py's CPU legs
use this module, as the checker and the timed CPU baseline.

* ``ray_table`` restates make_ray_projections and evaluate_sh16
  (vertex_baker/cpp/tinybvh_visibility.cpp:52-101) in numpy float32, with
  the C library's cosf/sinf, in the caster's operation order.
* ``visibility_sh16`` restates the caster's per-sample loop
  (tinybvh_visibility.cpp:145-230): origin = position + normalize(normal) *
  self_bias, or the (0,0,1) normal and a one-float nudge towards each ray
  when the normal is zero or non-finite (:103-137); each ray is an any-hit
  query in [0, max_distance] -- here the oracle's own watertight any-hit
  (``OracleScene.visibility``, float mode, the GPU's bit-exact twin); the
  unoccluded rays' weighted SH are summed per 64-ray batch in ray order and
  the batches added to the total.
* ``ReferenceCaster`` loads the caster compiled from the reference's sources
  into oracle/_ref/ (see oracle/Makefile) and calls
  vbake_pmr_visibility_sh_tinybvh (vertex_baker/cpp/vertex_baking_utils.h:73-90).
* ``compare`` is the comparison of the reference's benchmark
  (vertex_baker/benchmark_tinybvh_visibility.py:45-61): per-sample visible
  counts recovered from SH0, and SH differences.
"""

from __future__ import annotations

import ctypes
import ctypes.util
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BATCH = 64

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.cosf.restype = ctypes.c_float
_libm.cosf.argtypes = [ctypes.c_float]
_libm.sinf.restype = ctypes.c_float
_libm.sinf.argtypes = [ctypes.c_float]


def _reverse_bits(v: int) -> int:
    return int(f"{v:032b}"[::-1], 2)


def ray_table(ray_count: int) -> np.ndarray:
    """f32[R, 20]: direction xyz, 0, the 16 weighted SH values of each ray."""
    f = np.float32
    pi = f(3.14159265358979323846)
    weight = (f(4.0) * pi) / f(ray_count)
    out = np.zeros((ray_count, 20), np.float32)
    for r in range(ray_count):
        u0 = f(r) / f(ray_count)
        u1 = f(_reverse_bits(r)) * f(2.3283064365386963e-10)
        phi = u0 * (f(2.0) * pi)
        ct = f(1.0) - f(2.0) * u1
        st = np.sqrt(max(f(1.0) - ct * ct, f(0.0)), dtype=np.float32)
        x = f(_libm.cosf(float(phi))) * st
        y = ct
        z = f(_libm.sinf(float(phi))) * st
        x2, y2, z2 = x * x, y * y, z * z
        sh = [
            weight * f(0.282094791774),
            weight * (f(-0.488602511903) * y),
            weight * (f(0.488602511903) * z),
            weight * (f(-0.488602511903) * x),
            weight * (f(1.09254843059) * x * y),
            weight * (f(-1.09254843059) * y * z),
            weight * (f(0.315391565253) * (f(-1.0) + f(3.0) * z2)),
            weight * (f(-1.09254843059) * x * z),
            weight * (f(0.546274215296) * (x2 - y2)),
            weight * (f(-0.590043589927) * (f(3.0) * x2 * y - y2 * y)),
            weight * (f(2.89061144264) * x * y * z),
            weight * (f(-0.457045799464) * y * (f(-1.0) + f(5.0) * z2)),
            weight * (f(0.37317633259) * z * (f(-3.0) + f(5.0) * z2)),
            weight * (f(-0.457045799464) * x * (f(-1.0) + f(5.0) * z2)),
            weight * (f(1.44530572132) * (x2 - y2) * z),
            weight * (f(-0.590043589927) * (x2 * x - f(3.0) * x * y2)),
        ]
        out[r, 0:3] = (x, y, z)
        out[r, 4:] = np.array(sh, dtype=np.float32)
    return out


def ray_origins(positions: np.ndarray, normals: np.ndarray, self_bias: float):
    """(origins f32[S,3], has_normal bool[S]) of the caster's samples."""
    p = np.ascontiguousarray(positions, np.float32)
    n = np.ascontiguousarray(normals, np.float32)
    ls = (n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]) + n[:, 2] * n[:, 2]
    has = np.isfinite(ls) & (ls > np.float32(1e-16))
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        inv = np.float32(1.0) / np.sqrt(ls)
        u = np.where(has[:, None], n * inv[:, None], np.array([0.0, 0.0, 1.0], np.float32)).astype(np.float32)
    bias = np.float32(max(0.0, float(self_bias)))
    return (p + u * bias).astype(np.float32), has


def visibility_masks(orc, positions, normals, table, max_distance: float, self_bias: float) -> np.ndarray:
    """bool[S, R]: ray r of sample s is unoccluded, by the oracle's any-hit."""
    o, has = ray_origins(positions, normals, self_bias)
    d = table[:, 0:3]
    s_count, r_count = o.shape[0], d.shape[0]
    oo = np.broadcast_to(o[:, None, :], (s_count, r_count, 3)).copy()
    nudge = ~has
    if nudge.any():
        dd = np.broadcast_to(d[None], (int(nudge.sum()), r_count, 3))
        base = oo[nudge]
        up = np.nextafter(base, np.float32(np.inf))
        down = np.nextafter(base, np.float32(-np.inf))
        oo[nudge] = np.where(dd > 0, up, np.where(dd < 0, down, base))
    tmax = np.float32(max_distance) if np.isfinite(max_distance) and max_distance > 0 else np.float32(1e30)
    rays = np.zeros((s_count * r_count, 8), np.float32)
    rays[:, 0:3] = oo.reshape(-1, 3)
    rays[:, 4:7] = np.broadcast_to(d[None], (s_count, r_count, 3)).reshape(-1, 3)
    rays[:, 7] = tmax
    vis, _ = orc.visibility(rays)
    return (vis.reshape(s_count, r_count) > 0.5)


def sum_sh16(masks: np.ndarray, table: np.ndarray) -> np.ndarray:
    """The caster's SH sum: per 64-ray batch in ray order, then batch into total."""
    s_count, r_count = masks.shape
    total = np.zeros((s_count, 16), np.float32)
    for b in range(0, r_count, BATCH):
        batch = np.zeros((s_count, 16), np.float32)
        for r in range(b, min(b + BATCH, r_count)):
            batch = np.where(masks[:, r:r + 1], batch + table[r, 4:], batch).astype(np.float32)
        total = (total + batch).astype(np.float32)
    return total


def visibility_sh16(orc, positions, normals, ray_count: int = 512, max_distance: float = 0.5,
                    self_bias: float = 0.001):
    """(sh16 f32[S,16], visible counts i64[S]) of the caster's loop on the oracle."""
    table = ray_table(ray_count)
    masks = visibility_masks(orc, positions, normals, table, max_distance, self_bias)
    return sum_sh16(masks, table), masks.sum(axis=1)


class ReferenceCaster:
    """The reference's own caster, compiled from its sources into oracle/_ref/."""

    def __init__(self, layout: str = "bvh8"):
        names = {"bvh8": ["libvbake_bvh8.so", "libvbake_bvh.so"], "bvh": ["libvbake_bvh.so"]}[layout]
        self.lib = None
        for name in names:
            path = HERE / "_ref" / name
            if path.exists():
                lib = ctypes.CDLL(str(path))
                lib.vbake_tinybvh_has_bvh8_cpu.restype = ctypes.c_int
                lib.vbake_pmr_visibility_sh_tinybvh.restype = ctypes.c_int
                lib.vbake_last_error.restype = ctypes.c_char_p
                self.lib, self.name = lib, name
                self.layout = 1 if (layout == "bvh8" and lib.vbake_tinybvh_has_bvh8_cpu()) else 0
                break

    @property
    def available(self) -> bool:
        return self.lib is not None

    def cast(self, positions, indices, sites, normals, ray_count=512, max_distance=0.5, self_bias=1e-3,
             thread_count=0):
        """(sh16 f32[S,16], stats) of vbake_pmr_visibility_sh_tinybvh."""
        vp = ctypes.c_void_p
        positions = np.ascontiguousarray(positions, np.float32)
        indices = np.ascontiguousarray(indices, np.uint32)
        sites = np.ascontiguousarray(sites, np.float32)
        normals = np.ascontiguousarray(normals, np.float32)
        out = np.zeros((sites.shape[0], 16), np.float32)
        build_ms, trace_ms = ctypes.c_double(), ctypes.c_double()
        visible, threads = ctypes.c_ulonglong(), ctypes.c_int()
        rc = self.lib.vbake_pmr_visibility_sh_tinybvh(
            ctypes.c_int(positions.shape[0]), ctypes.c_int(indices.shape[0]), vp(positions.ctypes.data),
            vp(indices.ctypes.data), ctypes.c_int(sites.shape[0]), vp(sites.ctypes.data), vp(normals.ctypes.data),
            ctypes.c_int(ray_count), ctypes.c_float(max_distance), ctypes.c_float(self_bias),
            ctypes.c_int(thread_count), ctypes.c_int(self.layout), vp(out.ctypes.data), ctypes.byref(build_ms),
            ctypes.byref(trace_ms), ctypes.byref(visible), ctypes.byref(threads))
        if rc != 0:
            raise RuntimeError(self.lib.vbake_last_error().decode())
        return out, {"trace_ms": trace_ms.value, "build_ms": build_ms.value, "visible": int(visible.value),
                     "threads": int(threads.value), "layout": "BVH8_CPU" if self.layout == 1 else "BVH",
                     "library": self.name}


def world_geometry(world_triangles: np.ndarray):
    """positions f32[3T,3], indices u32[T,3] of world triangles f32[T,9]."""
    t = np.ascontiguousarray(world_triangles, np.float32).reshape(-1, 9)
    return t.reshape(-1, 3).copy(), np.arange(3 * t.shape[0], dtype=np.uint32).reshape(-1, 3)


def compare(reference: np.ndarray, candidate: np.ndarray, ray_count: int) -> dict:
    diff = candidate.astype(np.float64) - reference.astype(np.float64)
    per_ray = 0.282094791774 * (4.0 * np.pi / float(ray_count))
    ref_counts = np.rint(reference[:, 0] / per_ray).astype(np.int64)
    cand_counts = np.rint(candidate[:, 0] / per_ray).astype(np.int64)
    dc = np.abs(cand_counts - ref_counts)
    ad = np.abs(diff)
    return {"samples": int(reference.shape[0]), "mean_abs_sh": float(ad.mean()), "max_abs_sh": float(ad.max()),
            "rms_sh": float(np.sqrt(np.mean(diff * diff))),
            "samples_with_visible_count_difference": int(np.count_nonzero(dc)),
            "samples_with_exact_visible_count": int(np.count_nonzero(dc == 0)),
            "max_visible_count_difference": int(dc.max()),
            "samples_with_identical_sh16": int(np.count_nonzero(np.all(candidate == reference, axis=1)))}
