"""ctypes binding of the reference's own probe-placement library.

TEST INFRASTRUCTURE ONLY. ``_ref/libsurface_probe_sampler.so`` is compiled by
``oracle/Makefile`` straight from the reference's ``surface_probe_sampler.cpp``
(and its vendored cyCodeBase headers) where they lie; nothing of it is copied
into this repository and the product package never loads it. The tests call
its C ABI (surface_probe_sampler.h:120-223) to pin the oracle and the GPU
placement passes against the reference's default (C++) sampler backend.

``available()`` is False where the library was not built (a checkout without
the reference tree and without the prebuilt file).
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libsurface_probe_sampler.so"

_u32p = ctypes.POINTER(ctypes.c_uint32)
_f32p = ctypes.POINTER(ctypes.c_float)


class WSEOptions(ctypes.Structure):
    _fields_ = [("surface_area", ctypes.c_float), ("normal_cosine_threshold", ctypes.c_float),
                ("plane_distance_scale", ctypes.c_float)]


class AdaptiveWSEProfile(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "setup_ms", "stage1_partition_ms", "stage1_eliminate_wall_ms", "stage1_pack_cpu_ms", "stage1_grid_cpu_ms",
        "stage1_weights_cpu_ms", "stage1_heap_cpu_ms", "stage2_partition_ms", "stage2_eliminate_wall_ms",
        "stage2_pack_cpu_ms", "stage2_grid_cpu_ms", "stage2_weights_cpu_ms", "stage2_heap_cpu_ms", "final_pack_ms",
        "final_grid_ms", "final_weights_ms", "final_heap_ms", "total_ms")] + [(n, ctypes.c_uint32) for n in (
            "stage1_input_count", "stage1_output_count", "stage2_output_count", "final_output_count",
            "stage1_partition_count", "stage2_partition_count", "parallel_path")]


class RepairOptions(ctypes.Structure):
    _fields_ = [("min_gather_count", ctypes.c_uint32), ("max_repair_count", ctypes.c_uint32),
                ("normal_cosine_threshold", ctypes.c_float), ("weight_epsilon", ctypes.c_float)]


class SupportOptions(ctypes.Structure):
    _fields_ = [("normal_cosine_threshold", ctypes.c_float), ("weight_epsilon", ctypes.c_float),
                ("max_density_multiplier", ctypes.c_float)]


_LIB = None


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is not built (make -C oracle ref)")
        _LIB = ctypes.CDLL(str(LIB_PATH))
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f3(a):
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1, 3)


def _u(a):
    return np.ascontiguousarray(a, dtype=np.uint32).reshape(-1)


def _call(name, *args):
    err = ctypes.create_string_buffer(1024)
    fn = getattr(lib(), name)
    fn.restype = ctypes.c_int
    if not fn(*args, err, ctypes.c_size_t(len(err))):
        raise ValueError(err.value.decode())


def wse_eliminate(positions, normals, output_count, *, surface_area, normal_cosine_threshold=0.5,
                  plane_distance_scale=0.35):
    """surface_probe_wse_eliminate: (selected indices as the library returns
    them, Poisson radius)."""
    p, n = _f3(positions), _f3(normals)
    out = np.zeros(max(int(output_count), 1), np.uint32)
    radius = ctypes.c_float(0.0)
    opt = WSEOptions(float(surface_area), float(normal_cosine_threshold), float(plane_distance_scale))
    _call("surface_probe_wse_eliminate", _p(p), _p(n), ctypes.c_uint32(p.shape[0]), ctypes.c_uint32(int(output_count)),
          ctypes.byref(opt), _p(out), ctypes.byref(radius))
    return out[:int(output_count)], float(radius.value)


def wse_eliminate_adaptive(positions, normals, relative_densities, partition_masses, output_count, *, surface_area,
                           normal_cosine_threshold=0.5, plane_distance_scale=0.35):
    """surface_probe_wse_eliminate_adaptive: (selected indices, Poisson
    radius, profile)."""
    p, n = _f3(positions), _f3(normals)
    dens = np.ascontiguousarray(relative_densities, dtype=np.float32).reshape(-1)
    mass = np.ascontiguousarray(partition_masses, dtype=np.float32).reshape(-1)
    out = np.zeros(max(int(output_count), 1), np.uint32)
    radius = ctypes.c_float(0.0)
    prof = AdaptiveWSEProfile()
    opt = WSEOptions(float(surface_area), float(normal_cosine_threshold), float(plane_distance_scale))
    _call("surface_probe_wse_eliminate_adaptive", _p(p), _p(n), _p(dens), _p(mass), ctypes.c_uint32(p.shape[0]),
          ctypes.c_uint32(int(output_count)), ctypes.byref(opt), _p(out), ctypes.byref(radius), ctypes.byref(prof))
    return out[:int(output_count)], float(radius.value), prof


def deficit_repair(base_positions, base_normals, base_instances, candidate_positions, candidate_normals,
                   candidate_instances, audit_positions, audit_normals, audit_instances, instance_radii, *,
                   min_gather_count=4, max_repair_count=0, normal_cosine_threshold=0.5, weight_epsilon=1e-6):
    """surface_probe_deficit_repair: a dict like the oracle's."""
    bp, bn, bi = _f3(base_positions), _f3(base_normals), _u(base_instances)
    cp, cn, ci = _f3(candidate_positions), _f3(candidate_normals), _u(candidate_instances)
    ap, an, ai = _f3(audit_positions), _f3(audit_normals), _u(audit_instances)
    radii = np.ascontiguousarray(instance_radii, dtype=np.float32).reshape(-1)
    na = ap.shape[0]
    sel = np.zeros(max(1, cp.shape[0]), np.uint32)
    count = ctypes.c_uint32(0)
    out = {k: np.zeros(na, np.uint32) for k in ("counts_before", "counts_after")}
    out.update({k: np.zeros(na, np.float32) for k in ("weight_sums_before", "weight_sums_after", "ess_before",
                                                        "ess_after")})
    opt = RepairOptions(int(min_gather_count), int(max_repair_count), float(normal_cosine_threshold),
                        float(weight_epsilon))
    u = lambda v: ctypes.c_uint32(int(v))
    _call("surface_probe_deficit_repair", _p(bp), _p(bn), _p(bi), u(bp.shape[0]), _p(cp), _p(cn), _p(ci),
          u(cp.shape[0]), _p(ap), _p(an), _p(ai), u(na), _p(radii), u(radii.shape[0]), ctypes.byref(opt), _p(sel),
          ctypes.byref(count), _p(out["counts_before"]), _p(out["counts_after"]), _p(out["weight_sums_before"]),
          _p(out["weight_sums_after"]), _p(out["ess_before"]), _p(out["ess_after"]), ctypes.c_void_p(0))
    out["selected"] = sel[:count.value].astype(np.int64)
    return out


def filter_audit_repair_candidates(candidate_positions, candidate_normals, base_positions, base_normals,
                                   base_selected_indices, *, audit_cell_size, normal_cosine_threshold):
    """surface_probe_filter_audit_repair_candidates: (audit indices, repair
    indices), both ascending."""
    cp, cn = _f3(candidate_positions), _f3(candidate_normals)
    bp, bn = _f3(base_positions), _f3(base_normals)
    sel = _u(base_selected_indices)
    audit = np.zeros(max(cp.shape[0], 1), np.uint32)
    repair = np.zeros(max(cp.shape[0], 1), np.uint32)
    na, nr = ctypes.c_uint32(0), ctypes.c_uint32(0)
    u = lambda v: ctypes.c_uint32(int(v))
    _call("surface_probe_filter_audit_repair_candidates", _p(cp), _p(cn), u(cp.shape[0]), _p(bp), _p(bn),
          u(bp.shape[0]), _p(sel) if sel.size else ctypes.c_void_p(0), u(sel.shape[0]),
          ctypes.c_double(float(audit_cell_size)), ctypes.c_double(float(normal_cosine_threshold)), _p(audit),
          ctypes.byref(na), _p(repair), ctypes.byref(nr), ctypes.c_void_p(0))
    return audit[:na.value].astype(np.int64), repair[:nr.value].astype(np.int64)


def estimate_support(reference_positions, reference_normals, reference_instances, reference_area_weights,
                     query_positions, query_normals, query_instances, instance_radii, *, normal_cosine_threshold=0.5,
                     weight_epsilon=1e-6, max_density_multiplier=8.0):
    """surface_probe_estimate_support: (support f, density m)."""
    rp, rn, ri = _f3(reference_positions), _f3(reference_normals), _u(reference_instances)
    ra = np.ascontiguousarray(reference_area_weights, dtype=np.float32).reshape(-1)
    qp, qn, qi = _f3(query_positions), _f3(query_normals), _u(query_instances)
    radii = np.ascontiguousarray(instance_radii, dtype=np.float32).reshape(-1)
    f = np.zeros(qp.shape[0], np.float32)
    m = np.zeros(qp.shape[0], np.float32)
    opt = SupportOptions(float(normal_cosine_threshold), float(weight_epsilon), float(max_density_multiplier))
    u = lambda v: ctypes.c_uint32(int(v))
    _call("surface_probe_estimate_support", _p(rp), _p(rn), _p(ri), _p(ra), u(rp.shape[0]), _p(qp), _p(qn), _p(qi),
          u(qp.shape[0]), _p(radii), u(radii.shape[0]), ctypes.byref(opt), _p(f), _p(m))
    return f, m


class PointOctreeResult(ctypes.Structure):
    _fields_ = [("nodes", ctypes.POINTER(ctypes.c_uint32)), ("node_count", ctypes.c_uint32),
                ("probe_order", ctypes.POINTER(ctypes.c_uint32)), ("probe_count", ctypes.c_uint32),
                ("root_center", ctypes.c_double * 3), ("root_extent", ctypes.c_double)]


def build_point_octree(positions, *, leaf_capacity=8, max_depth=16):
    """surface_probe_build_point_octree: (nodes u32[M, 4], order i64[N],
    root centre, root half extent); the library's buffers are released."""
    p = _f3(positions)
    res = PointOctreeResult()
    u = lambda v: ctypes.c_uint32(int(v))
    _call("surface_probe_build_point_octree", _p(p), u(p.shape[0]), u(leaf_capacity), u(max_depth),
          ctypes.byref(res), ctypes.c_void_p(0))
    try:
        nodes = np.ctypeslib.as_array(res.nodes, shape=(res.node_count * 4,)).reshape(-1, 4).copy()
        order = np.ctypeslib.as_array(res.probe_order, shape=(res.probe_count,)).astype(np.int64)
        center = tuple(float(v) for v in res.root_center)
        extent = float(res.root_extent)
    finally:
        free = lib().surface_probe_free_point_octree
        free.restype = None
        free(ctypes.byref(res))
    return nodes, order, center, extent
