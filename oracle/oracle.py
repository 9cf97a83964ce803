"""ctypes binding of the CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY. The oracle is the checker for the CUDA path; the
product package ``nan_b200`` never imports this module. ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg are its only
users.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

F32 = 0
F64 = 1


class OracleLighting(ctypes.Structure):
    _fields_ = [
        ("sun_direction", ctypes.c_float * 3),
        ("sun_cos_half_angle", ctypes.c_float),
        ("sun_color", ctypes.c_float * 3),
        ("sun_intensity", ctypes.c_float),
        ("sun_transmittance", ctypes.c_float * 3),
        ("ray_t_max", ctypes.c_float),
        ("sky_radiance", ctypes.c_float * 3),
        ("flags", ctypes.c_uint32),
        ("sky_view_lut", ctypes.c_void_p),
        ("sky_view_width", ctypes.c_uint32),
        ("sky_view_height", ctypes.c_uint32),
        ("sky_view_up", ctypes.c_float * 3),
        ("sky_view_horizon_angle", ctypes.c_float),
    ]


class OracleProbeResolveOptions(ctypes.Structure):
    _fields_ = [
        ("debug_view", ctypes.c_uint32),
        ("min_gather_count", ctypes.c_uint32),
        ("use_vertex_fallback", ctypes.c_uint32),
        ("use_vertex_lighting", ctypes.c_uint32),
        ("use_radial_visibility", ctypes.c_uint32),
        ("frame_index", ctypes.c_uint32),
        ("max_density_multiplier", ctypes.c_float),
        ("vertex_lighting_rgbm_range", ctypes.c_float),
        ("vertex_lighting_rgbm", ctypes.c_void_p),
        ("vertex_lighting_target", ctypes.c_void_p),
        ("vertex_lighting_triangle_map", ctypes.c_void_p),
        ("vertex_lighting_instance_offsets", ctypes.c_void_p),
        ("vertex_lighting_vertex_count", ctypes.c_uint32),
        ("vertex_lighting_triangle_record_count", ctypes.c_uint32),
    ]


class OracleCamera(ctypes.Structure):
    _fields_ = [
        ("position", ctypes.c_float * 3),
        ("jitter_x", ctypes.c_float),
        ("image_u", ctypes.c_float * 3),
        ("jitter_y", ctypes.c_float),
        ("image_v", ctypes.c_float * 3),
        ("near_clip", ctypes.c_float),
        ("image_w", ctypes.c_float * 3),
        ("far_clip", ctypes.c_float),
    ]


class OracleRayCounts(ctypes.Structure):
    _fields_ = [
        ("extend_rays", ctypes.c_uint64),
        ("shadow_rays", ctypes.c_uint64),
        ("node_fetches", ctypes.c_uint64),
        ("triangle_tests", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


def build() -> Path:
    """Compile liboracle.so (and, where the reference tree exists, _ref/)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


def _p(array: np.ndarray):
    return array.ctypes.data_as(ctypes.c_void_p)


def _declare(l: ctypes.CDLL) -> None:
    vp, i, u32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32
    l.oracle_last_error.restype = ctypes.c_char_p
    l.oracle_rng_sequence.argtypes = [u32, u32, u32, i, vp]
    l.oracle_sincos.argtypes = [vp, i, vp, vp]
    l.oracle_atan2_asin.argtypes = [vp, vp, i, vp, vp]
    l.oracle_sky_radiance.argtypes = [ctypes.POINTER(OracleLighting), vp, i, i, vp]
    l.oracle_pack_rgb9e5.argtypes = [vp, i, vp]
    l.oracle_unpack_rgb9e5.argtypes = [vp, i, vp]
    l.oracle_f32_to_f16.argtypes = [vp, i, vp]
    l.oracle_hemi_oct_encode.argtypes = [vp, i, vp]
    l.oracle_hemi_oct_decode.argtypes = [vp, i, vp]
    l.oracle_cosine_sample_hemisphere.argtypes = [vp, i, vp]
    l.oracle_mesh_colors_address_to_ij.argtypes = [vp, vp, i, vp]
    l.oracle_scene_create.restype = vp
    l.oracle_scene_create.argtypes = [vp, i, vp, i, vp, i, vp, i, vp, vp, i, vp, i]
    l.oracle_scene_destroy.argtypes = [vp]
    l.oracle_scene_triangle_count.argtypes = [vp]
    l.oracle_scene_world_triangles.argtypes = [vp, vp]
    l.oracle_scene_bvh_stats.argtypes = [vp, vp]
    l.oracle_sah_build_stats.argtypes = [vp, ctypes.c_uint32, vp]
    l.oracle_intersect.argtypes = [vp, vp, i, i, vp, vp, vp]
    l.oracle_visibility.argtypes = [vp, vp, i, i, vp, vp]
    l.oracle_trace_screen.argtypes = [vp, vp, vp, u32, u32, u32, u32, vp, i, i, i, vp, vp]
    l.oracle_trace_texels.argtypes = [vp, vp, vp, u32, vp, u32, vp, vp, u32, vp, i,
                                      u32, u32, u32, i, i, i, vp]
    l.oracle_trace_probes.argtypes = [vp, vp, vp, vp, vp, vp, vp, u32, vp, u32, vp, i,
                                      u32, u32, u32, i, i, i, vp]
    l.oracle_trace_probes_independent.argtypes = l.oracle_trace_probes.argtypes
    l.oracle_scene_set_area_lights.argtypes = [vp, vp, i, ctypes.c_float]
    l.oracle_resolve_probes.argtypes = [vp, vp, vp, u32, u32, vp, i, vp, u32, vp, u32, vp, u32, vp, u32, vp, vp, vp,
                                        vp, vp, i, vp]
    l.oracle_wse_eliminate.argtypes = [vp, vp, vp, vp, u32, vp, vp, ctypes.c_float, ctypes.c_float, vp, vp, vp, i]
    l.oracle_deficit_repair.argtypes = [vp, vp, vp, u32, vp, vp, vp, u32, vp, vp, vp, u32, vp, u32, u32, u32,
                                        ctypes.c_float, ctypes.c_float, vp, vp, vp, vp, vp, vp, vp, vp]
    l.oracle_filter_audit_repair.argtypes = [vp, vp, vp, u32, vp, vp, vp, u32, vp, u32, u32, vp, ctypes.c_double,
                                             vp, ctypes.POINTER(ctypes.c_uint32), vp,
                                             ctypes.POINTER(ctypes.c_uint32)]
    l.oracle_estimate_support.argtypes = [vp, vp, vp, vp, u32, vp, vp, vp, u32, vp, u32, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_float, vp, vp]
    l.own_exp.argtypes = [ctypes.c_float]
    l.own_exp.restype = ctypes.c_float
    l.own_log2.argtypes = [ctypes.c_float]
    l.own_log2.restype = ctypes.c_float
    l.oracle_prt_project_lighting.argtypes = [vp, u32, vp]
    l.oracle_prt_project_lighting.restype = None
    l.oracle_prt_evaluate.argtypes = [vp, vp, vp, vp, vp, vp, u32]
    l.oracle_prt_evaluate.restype = None
    l.oracle_trace_probes_prt.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, u32, vp, vp, i, u32, u32, u32, i, i, i]
    l.oracle_filter_mesh_colors.argtypes = [vp, vp, vp, u32, vp, vp, vp, vp, ctypes.c_float, ctypes.c_float, i]
    l.oracle_resolve_mesh_colors.argtypes = [vp, vp, vp, u32, u32, vp, i, vp, vp, vp, u32, vp, i, i, i, vp]
    l.oracle_trace_points.argtypes = [vp, vp, vp, i, u32, u32, u32, u32, vp, i, i, vp]


# ---- scalar helpers --------------------------------------------------------
def filter_mesh_colors(face_infos, instance_infos, side_infos, adjacency, face_normals, source, neighbor_weight,
                       normal_sigma_radians, threads=0):
    """One surface-filter pass; source and the returned slots are uint32 [P, 4]."""
    fi = np.ascontiguousarray(face_infos, dtype=np.uint32).reshape(-1, 2)
    ii = np.ascontiguousarray(instance_infos, dtype=np.uint32).reshape(-1, 4)
    si = np.ascontiguousarray(side_infos, dtype=np.uint32).reshape(-1, 2)
    adj = np.ascontiguousarray(adjacency, dtype=np.uint32).reshape(-1, 4)
    nrm = np.ascontiguousarray(face_normals, dtype=np.float32).reshape(-1, 4)
    src = np.ascontiguousarray(source).view(np.uint32).reshape(-1, 4)
    dst = src.copy()
    lib().oracle_filter_mesh_colors(_p(fi), _p(ii), _p(si), ii.shape[0], _p(adj), _p(nrm), _p(src), _p(dst),
                                    float(neighbor_weight), float(normal_sigma_radians), threads)
    return dst


def wse_eliminate(positions, normals, set_offsets, output_counts, surface_areas, normal_cosine_threshold=0.5,
                  plane_distance_scale=0.35, threads=0, relative_densities=None):
    """Sequential weighted sample elimination per contiguous set; returns
    (keep u8[N], poisson radii f32[S], removal order u32[N] per set from its
    first slot, ~0 past the eliminated ones). relative_densities (f32[N])
    selects the adaptive elimination."""
    p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    dens = None if relative_densities is None else np.ascontiguousarray(relative_densities,
                                                                         dtype=np.float32).reshape(-1)
    nrm = np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
    off = np.ascontiguousarray(set_offsets, dtype=np.uint32).reshape(-1)
    outs = np.ascontiguousarray(output_counts, dtype=np.uint32).reshape(-1)
    areas = np.ascontiguousarray(surface_areas, dtype=np.float32).reshape(-1)
    keep = np.zeros(p.shape[0], np.uint8)
    radii = np.zeros(outs.shape[0], np.float32)
    order = np.full(p.shape[0], 0xFFFFFFFF, np.uint32)
    rc = lib().oracle_wse_eliminate(_p(p), _p(nrm), None if dens is None else _p(dens), _p(off), outs.shape[0],
                                    _p(outs), _p(areas),
                                    float(normal_cosine_threshold), float(plane_distance_scale), _p(keep),
                                    _p(radii), _p(order), threads)
    if rc != 0:
        raise RuntimeError("weighted sample elimination: a candidate has more than 8000 neighbours")
    return keep, radii, order


def deficit_repair(base_positions, base_normals, base_instances, candidate_positions, candidate_normals,
                   candidate_instances, audit_positions, audit_normals, audit_instances, instance_radii, *,
                   min_gather_count=4, max_repair_count=0, normal_cosine_threshold=0.5, weight_epsilon=1e-6):
    """One-at-a-time deficit repair; returns a dict with selected (choice
    order), counts/weight sums/ess before and after."""
    def arrays(p, n, i):
        return (np.ascontiguousarray(p, dtype=np.float32).reshape(-1, 3),
                np.ascontiguousarray(n, dtype=np.float32).reshape(-1, 3),
                np.ascontiguousarray(i, dtype=np.uint32).reshape(-1))
    bp, bn, bi = arrays(base_positions, base_normals, base_instances)
    cp, cn, ci = arrays(candidate_positions, candidate_normals, candidate_instances)
    ap, an, ai = arrays(audit_positions, audit_normals, audit_instances)
    radii = np.ascontiguousarray(instance_radii, dtype=np.float32).reshape(-1)
    na = ap.shape[0]
    sel = np.zeros(max(1, min(int(max_repair_count), cp.shape[0])), np.uint32)
    count = ctypes.c_uint32(0)
    out = {k: np.zeros(na, np.uint32) for k in ("counts_before", "counts_after")}
    out.update({k: np.zeros(na, np.float32) for k in ("weight_sums_before", "weight_sums_after", "ess_before",
                                                        "ess_after")})
    rc = lib().oracle_deficit_repair(_p(bp), _p(bn), _p(bi), bp.shape[0], _p(cp), _p(cn), _p(ci), cp.shape[0],
                                     _p(ap), _p(an), _p(ai), na, _p(radii), radii.shape[0], int(min_gather_count),
                                     int(max_repair_count), float(normal_cosine_threshold), float(weight_epsilon),
                                     _p(sel), ctypes.byref(count), _p(out["counts_before"]), _p(out["counts_after"]),
                                     _p(out["weight_sums_before"]), _p(out["weight_sums_after"]),
                                     _p(out["ess_before"]), _p(out["ess_after"]))
    if rc != 0:
        raise RuntimeError("deficit repair: an audit names an instance out of range")
    out["selected"] = sel[:count.value].astype(np.int64)
    return out


def filter_audit_repair(candidate_positions, candidate_normals, base_positions, base_normals, base_selected_indices,
                        *, audit_cell_size, normal_cosine_threshold, candidate_sets=None, base_sets=None):
    """(audit indices, repair indices), int64 ascending."""
    cp = np.ascontiguousarray(candidate_positions, dtype=np.float32).reshape(-1, 3)
    cn = np.ascontiguousarray(candidate_normals, dtype=np.float32).reshape(-1, 3)
    bp = np.ascontiguousarray(base_positions, dtype=np.float32).reshape(-1, 3)
    bn = np.ascontiguousarray(base_normals, dtype=np.float32).reshape(-1, 3)
    sel = np.ascontiguousarray(base_selected_indices, dtype=np.uint32).reshape(-1)
    cells = np.ascontiguousarray(np.atleast_1d(np.asarray(audit_cell_size, dtype=np.float64)))
    cs = None if candidate_sets is None else np.ascontiguousarray(candidate_sets, dtype=np.uint32).reshape(-1)
    bs = None if base_sets is None else np.ascontiguousarray(base_sets, dtype=np.uint32).reshape(-1)
    audit = np.zeros(max(cp.shape[0], 1), np.uint32)
    repair = np.zeros(max(cp.shape[0], 1), np.uint32)
    na, nr = ctypes.c_uint32(0), ctypes.c_uint32(0)
    rc = lib().oracle_filter_audit_repair(_p(cp), _p(cn), None if cs is None else _p(cs), cp.shape[0], _p(bp), _p(bn),
                                          None if bs is None else _p(bs), bp.shape[0], _p(sel), sel.shape[0],
                                          cells.shape[0], _p(cells), float(normal_cosine_threshold), _p(audit),
                                          ctypes.byref(na), _p(repair), ctypes.byref(nr))
    if rc:
        raise ValueError("base_selected_indices contains an invalid index" if rc == 1 else
                         "a candidate set index is out of range")
    return audit[:na.value].astype(np.int64), repair[:nr.value].astype(np.int64)


def estimate_support(reference_positions, reference_normals, reference_instances, reference_area_weights,
                     query_positions, query_normals, query_instances, instance_radii, *, normal_cosine_threshold=0.5,
                     weight_epsilon=1e-6, max_density_multiplier=8.0):
    """Support f and density m per query site (float32 each)."""
    rp = np.ascontiguousarray(reference_positions, dtype=np.float32).reshape(-1, 3)
    rn = np.ascontiguousarray(reference_normals, dtype=np.float32).reshape(-1, 3)
    ri = np.ascontiguousarray(reference_instances, dtype=np.uint32).reshape(-1)
    ra = np.ascontiguousarray(reference_area_weights, dtype=np.float32).reshape(-1)
    qp = np.ascontiguousarray(query_positions, dtype=np.float32).reshape(-1, 3)
    qn = np.ascontiguousarray(query_normals, dtype=np.float32).reshape(-1, 3)
    qi = np.ascontiguousarray(query_instances, dtype=np.uint32).reshape(-1)
    radii = np.ascontiguousarray(instance_radii, dtype=np.float32).reshape(-1)
    f = np.zeros(qp.shape[0], np.float32)
    m = np.zeros(qp.shape[0], np.float32)
    rc = lib().oracle_estimate_support(_p(rp), _p(rn), _p(ri), _p(ra), rp.shape[0], _p(qp), _p(qn), _p(qi),
                                       qp.shape[0], _p(radii), radii.shape[0], float(normal_cosine_threshold),
                                       float(weight_epsilon), float(max_density_multiplier), _p(f), _p(m))
    if rc != 0:
        raise RuntimeError("support estimate: an instance index is out of range")
    return f, m


def sah_build_stats(world_triangles) -> dict:
    """The library's default BVH builder (binned SAH, 32 bins, then the SAH
    leaf collapse of up to 3 triangles) restated on the CPU: its kept interior
    node count and SAH cost for world triangles f32[T, 9] in flattened order."""
    w = np.ascontiguousarray(world_triangles, dtype=np.float32).reshape(-1, 9)
    out = np.zeros(3, np.float64)
    lib().oracle_sah_build_stats(_p(w), w.shape[0], _p(out))
    return {"nodes": int(out[0]), "sah_cost": float(out[2])}


def own_exp(x: float) -> float:
    """The kernels' own float e^x (nan_exp)."""
    return float(lib().own_exp(float(x)))


def own_log2(x: float) -> float:
    """The kernels' own float log2 (nan_log2)."""
    return float(lib().own_log2(float(x)))


def prt_project_lighting(lighting, sample_count=2048):
    """SH L2 projection of the escape radiance, f32[9, 4]."""
    sh = np.zeros((9, 4), np.float32)
    L = lighting_struct(lighting)
    lib().oracle_prt_project_lighting(ctypes.byref(L), int(sample_count), _p(sh))
    return sh


def prt_evaluate(values, sample_counts, static_source, sh):
    """Evaluated irradiance f32[N, 3] and the copied counts u32[N]."""
    v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1, 27)
    c = np.ascontiguousarray(sample_counts).view(np.uint32).reshape(-1)
    st = np.ascontiguousarray(static_source, dtype=np.float32).reshape(-1, 3)
    s = np.ascontiguousarray(sh, dtype=np.float32).reshape(9, 4)
    out = np.zeros((v.shape[0], 3), np.float32)
    counts = np.zeros(v.shape[0], np.uint32)
    lib().oracle_prt_evaluate(_p(v), _p(c), _p(st), _p(s), _p(out), _p(counts), v.shape[0])
    return out, counts



def rng_sequence(x: int, y: int, sample_index: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.float32)
    lib().oracle_rng_sequence(x, y, sample_index, count, _p(out))
    return out


def atan2_asin(y: np.ndarray, x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The kernels' own atan2(y, x) and asin(y), float32."""
    yy = np.ascontiguousarray(y, dtype=np.float32)
    xx = np.ascontiguousarray(x, dtype=np.float32)
    a = np.zeros_like(yy)
    s = np.zeros_like(yy)
    lib().oracle_atan2_asin(_p(yy), _p(xx), yy.size, _p(a), _p(s))
    return a, s


def sky_radiance(lighting, dirs: np.ndarray, precision: int = F32) -> np.ndarray:
    """sample_sky_lut of `lighting` (a NanLighting-like object) for unit directions f32[N, 3]."""
    d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
    out = np.zeros_like(d)
    s = lighting_struct(lighting)
    lib().oracle_sky_radiance(ctypes.byref(s), _p(d), d.shape[0], precision, _p(out))
    return out


def sincos(angles: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    a = np.ascontiguousarray(angles, dtype=np.float32)
    s = np.zeros_like(a)
    c = np.zeros_like(a)
    lib().oracle_sincos(_p(a), a.size, _p(s), _p(c))
    return s, c


def pack_rgb9e5(rgb: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(rgb, dtype=np.float32).reshape(-1, 3)
    out = np.zeros(v.shape[0], dtype=np.uint32)
    lib().oracle_pack_rgb9e5(_p(v), v.shape[0], _p(out))
    return out


def unpack_rgb9e5(packed: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(packed, dtype=np.uint32).reshape(-1)
    out = np.zeros((p.size, 3), dtype=np.float32)
    lib().oracle_unpack_rgb9e5(_p(p), p.size, _p(out))
    return out


def f32_to_f16(values: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
    out = np.zeros(v.size, dtype=np.uint16)
    lib().oracle_f32_to_f16(_p(v), v.size, _p(out))
    return out


def hemi_oct_encode(dirs: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
    out = np.zeros((d.shape[0], 2), dtype=np.float32)
    lib().oracle_hemi_oct_encode(_p(d), d.shape[0], _p(out))
    return out


def hemi_oct_decode(uv: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(uv, dtype=np.float32).reshape(-1, 2)
    out = np.zeros((u.shape[0], 3), dtype=np.float32)
    lib().oracle_hemi_oct_decode(_p(u), u.shape[0], _p(out))
    return out


def cosine_sample_hemisphere(u: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(u, dtype=np.float32).reshape(-1, 2)
    out = np.zeros((a.shape[0], 4), dtype=np.float32)
    lib().oracle_cosine_sample_hemisphere(_p(a), a.shape[0], _p(out))
    return out


def address_to_ij(address: np.ndarray, resolution: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(address, dtype=np.uint32)
    r = np.ascontiguousarray(resolution, dtype=np.uint32)
    out = np.zeros((a.size, 2), dtype=np.uint32)
    lib().oracle_mesh_colors_address_to_ij(_p(a), _p(r), a.size, _p(out))
    return out


# ---- scenes and integrators ------------------------------------------------

def lighting_struct(lighting) -> OracleLighting:
    """Build the C struct from any object with the NanLighting field names."""
    s = OracleLighting()
    s.sun_direction[:] = [float(x) for x in lighting.sun_direction]
    s.sun_cos_half_angle = float(lighting.sun_cos_half_angle)
    s.sun_color[:] = [float(x) for x in lighting.sun_color]
    s.sun_intensity = float(lighting.sun_intensity)
    s.sun_transmittance[:] = [float(x) for x in lighting.sun_transmittance]
    s.ray_t_max = float(lighting.ray_t_max)
    s.sky_radiance[:] = [float(x) for x in lighting.sky_radiance]
    s.flags = int(lighting.flags)
    lut = getattr(lighting, "sky_view_lut", None)
    if lut is not None:
        host = np.ascontiguousarray((lut.cpu().numpy() if hasattr(lut, "cpu") else lut), dtype=np.float32)
        s._sky_view_host = host  # keeps the host copy alive with the struct
        s.sky_view_lut = host.ctypes.data
        s.sky_view_height, s.sky_view_width = int(host.shape[0]), int(host.shape[1])
    s.sky_view_up[:] = [float(x) for x in getattr(lighting, "sky_view_up", (0.0, 1.0, 0.0))]
    horizon = getattr(lighting, "sky_view_horizon_angle", None)
    if horizon is None:
        # the reference atmosphere's view height (scene.slang:474), in float32
        h, r = np.float32(6.3602), np.float32(6.36)
        horizon = float(np.float32(np.arccos(np.sqrt(h * h - r * r) / h)) - np.float32(0.5) * np.float32(np.pi))
    s.sky_view_horizon_angle = float(horizon)
    return s


def camera_struct(camera) -> OracleCamera:
    c = OracleCamera()
    c.position[:] = [float(x) for x in camera.position]
    c.image_u[:] = [float(x) for x in camera.image_u]
    c.image_v[:] = [float(x) for x in camera.image_v]
    c.image_w[:] = [float(x) for x in camera.image_w]
    c.jitter_x = float(camera.jitter[0])
    c.jitter_y = float(camera.jitter[1])
    c.near_clip = float(camera.near_clip_plane)
    c.far_clip = float(camera.far_clip_plane)
    return c


class OracleScene:
    """CPU copy of a scene in the reference's record layouts."""

    def __init__(self, vertices, indices, mesh_descs, instance_descs, transforms,
                 inverse_transposes, materials):
        self._keep = [
            np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 8),
            np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3),
            np.ascontiguousarray(mesh_descs, dtype=np.uint32).reshape(-1, 4),
            np.ascontiguousarray(instance_descs, dtype=np.uint32).reshape(-1, 4),
            np.ascontiguousarray(transforms, dtype=np.float32).reshape(-1, 16),
            np.ascontiguousarray(inverse_transposes, dtype=np.float32).reshape(-1, 16),
            np.ascontiguousarray(materials, dtype=np.float32).reshape(-1, 8),
        ]
        v, ix, md, idesc, tr, it, mat = self._keep
        self.handle = lib().oracle_scene_create(
            _p(v), v.shape[0], _p(ix), ix.shape[0], _p(md), md.shape[0], _p(idesc),
            idesc.shape[0], _p(tr), _p(it), tr.shape[0], _p(mat), mat.shape[0])

    @classmethod
    def from_scene(cls, scene) -> "OracleScene":
        """From any object carrying the reference arrays as numpy/torch."""
        def a(x):
            return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)
        return cls(a(scene.vertices), a(scene.indices), a(scene.mesh_descs),
                   a(scene.instance_descs), a(scene.transforms),
                   a(scene.inverse_transposes), a(scene.materials))

    def __del__(self):
        if getattr(self, "handle", None):
            lib().oracle_scene_destroy(self.handle)
            self.handle = None

    @property
    def triangle_count(self) -> int:
        return int(lib().oracle_scene_triangle_count(self.handle))

    def world_triangles(self) -> np.ndarray:
        out = np.zeros((self.triangle_count, 9), dtype=np.float32)
        lib().oracle_scene_world_triangles(self.handle, _p(out))
        return out

    def bvh_stats(self) -> dict:
        out = np.zeros(3, dtype=np.float64)
        lib().oracle_scene_bvh_stats(self.handle, _p(out))
        return {"nodes": int(out[0]), "leaves": int(out[1]), "sah_cost": float(out[2])}

    def intersect(self, rays: np.ndarray, mode: int = 0):
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        ids = np.zeros((r.shape[0], 4), dtype=np.uint32)
        tb = np.zeros((r.shape[0], 3), dtype=np.float32)
        counts = OracleRayCounts()
        lib().oracle_intersect(self.handle, _p(r), r.shape[0], mode, _p(ids), _p(tb),
                               ctypes.byref(counts))
        return ids, tb, counts.as_dict()

    def visibility(self, rays: np.ndarray, mode: int = 0):
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        vis = np.zeros(r.shape[0], dtype=np.float32)
        counts = OracleRayCounts()
        lib().oracle_visibility(self.handle, _p(r), r.shape[0], mode, _p(vis),
                                ctypes.byref(counts))
        return vis, counts.as_dict()

    def trace_screen(self, lighting, camera, width, height, frame, max_vertices,
                     pixels, precision=F32, threads=0):
        px = np.ascontiguousarray(pixels, dtype=np.uint32).reshape(-1, 2)
        out = np.zeros((px.shape[0], 4), dtype=np.float32)
        counts = OracleRayCounts()
        L = lighting_struct(lighting)
        C = camera_struct(camera)
        rc = lib().oracle_trace_screen(self.handle, ctypes.byref(L), ctypes.byref(C),
                                       width, height, frame, max_vertices, _p(px),
                                       px.shape[0], precision, threads, _p(out),
                                       ctypes.byref(counts))
        if rc != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return out, counts.as_dict()

    def trace_texels(self, lighting, slots, face_infos, instance_infos, side_infos,
                     units, iteration, samples_per_texel, max_bounces, reset,
                     precision=F32, threads=0):
        """Updates ``slots`` (uint32 [P,4] or uint8 [P,16]) in place."""
        assert slots.flags["C_CONTIGUOUS"]
        fi = np.ascontiguousarray(face_infos, dtype=np.uint32).reshape(-1, 2)
        ii = np.ascontiguousarray(instance_infos, dtype=np.uint32).reshape(-1, 4)
        si = np.ascontiguousarray(side_infos, dtype=np.uint32).reshape(-1, 2)
        un = np.ascontiguousarray(units, dtype=np.uint32).reshape(-1, 2)
        counts = OracleRayCounts()
        L = lighting_struct(lighting)
        payload = slots.nbytes // 16
        rc = lib().oracle_trace_texels(self.handle, ctypes.byref(L), _p(slots), payload,
                                       _p(fi), fi.shape[0], _p(ii), _p(si), ii.shape[0],
                                       _p(un), un.shape[0], iteration, samples_per_texel,
                                       max_bounces, int(bool(reset)), precision, threads,
                                       ctypes.byref(counts))
        if rc != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return counts.as_dict()

    def resolve_mesh_colors(self, lighting, camera, width, height, pixels, face_infos, instance_infos, side_infos,
                            colors, packed=False, precision=F32, threads=0):
        """Mesh Colors resolve of pixels u32[N, 2]; colors are slots (uint32 [P, 4])
        or RGB9E5 words (uint32 [P]). Returns f32[N, 4]."""
        px = np.ascontiguousarray(pixels, dtype=np.uint32).reshape(-1, 2)
        fi = np.ascontiguousarray(face_infos, dtype=np.uint32).reshape(-1, 2)
        ii = np.ascontiguousarray(instance_infos, dtype=np.uint32).reshape(-1, 4)
        si = np.ascontiguousarray(side_infos, dtype=np.uint32).reshape(-1, 2)
        col = np.ascontiguousarray(colors, dtype=np.uint32)
        out = np.zeros((px.shape[0], 4), np.float32)
        L, C = lighting_struct(lighting), camera_struct(camera)
        rc = lib().oracle_resolve_mesh_colors(self.handle, ctypes.byref(L), ctypes.byref(C), width, height, _p(px),
                                              px.shape[0], _p(fi), _p(ii), _p(si), ii.shape[0], _p(col),
                                              int(bool(packed)), precision, threads, _p(out))
        if rc != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return out

    def resolve_probes(self, lighting, camera, width, height, pixels, layout, values, sample_counts, self_hits,
                       radial, *, debug_view=0, min_gather_count=4, use_radial_visibility=True,
                       use_vertex_fallback=False, frame_index=0, max_density_multiplier=8.0, threads=0):
        """Surface-probe resolve of pixels u32[N, 2] against a probe layout
        (probes, nodes, instance_gpu_data, triangle_vertex_probes) and an
        irradiance field; returns f32[N, 4]. Raises on an out-of-range index."""
        px = np.ascontiguousarray(pixels, dtype=np.uint32).reshape(-1, 2)
        pr = np.ascontiguousarray(layout.probes).view(np.float32).reshape(-1, 12)
        nd = np.ascontiguousarray(layout.nodes, dtype=np.uint32).reshape(-1, 4)
        ins = np.ascontiguousarray(layout.instance_gpu_data).view(np.float32).reshape(-1, 12)
        tm = np.ascontiguousarray(layout.triangle_vertex_probes, dtype=np.uint32).reshape(-1, 4)
        v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1, 3)
        c = np.ascontiguousarray(sample_counts).view(np.uint32).reshape(-1)
        sh = np.ascontiguousarray(self_hits).view(np.uint32).reshape(-1)
        rm = np.ascontiguousarray(radial).view(np.uint32).reshape(-1, 16)
        opt = OracleProbeResolveOptions(debug_view=int(debug_view), min_gather_count=int(min_gather_count),
                                        use_vertex_fallback=int(bool(use_vertex_fallback)),
                                        use_radial_visibility=int(bool(use_radial_visibility)),
                                        frame_index=int(frame_index) & 0xFFFFFFFF,
                                        max_density_multiplier=float(max_density_multiplier),
                                        vertex_lighting_rgbm_range=1.0)
        out = np.zeros((px.shape[0], 4), np.float32)
        L, C = lighting_struct(lighting), camera_struct(camera)
        rc = lib().oracle_resolve_probes(self.handle, ctypes.byref(L), ctypes.byref(C), width, height, _p(px),
                                         px.shape[0], _p(pr), pr.shape[0], _p(nd), nd.shape[0], _p(ins),
                                         ins.shape[0], _p(tm), tm.shape[0], _p(v), _p(c), _p(sh), _p(rm),
                                         ctypes.byref(opt), threads, _p(out))
        if rc != 0:
            raise RuntimeError("probe resolve: a layout index is out of range")
        return out

    def trace_probes_prt(self, lighting, values, sample_counts, self_hits, radial, static_source, probes,
                         probe_instances, units, iteration, samples_per_probe, max_bounces, reset, precision=F32,
                         threads=0):
        """PRT L2 baker; values f32[N, 27], static_source f32[N, 3] and the rest updated in place."""
        for buf in (values, sample_counts, self_hits, radial, static_source):
            assert buf.flags["C_CONTIGUOUS"]
        pr = np.ascontiguousarray(probes).view(np.uint8).reshape(-1)
        pi = np.ascontiguousarray(probe_instances).view(np.uint8).reshape(-1)
        un = np.ascontiguousarray(units, dtype=np.uint32).reshape(-1)
        L = lighting_struct(lighting)
        rc = lib().oracle_trace_probes_prt(self.handle, ctypes.byref(L), _p(values), _p(sample_counts),
                                           _p(self_hits), _p(radial), _p(static_source), _p(pr), pr.size // 48,
                                           _p(pi), _p(un), un.size, iteration, samples_per_probe, max_bounces,
                                           int(bool(reset)), precision, threads)
        if rc != 0:
            raise RuntimeError(lib().oracle_last_error().decode())

    def set_area_lights(self, lights, power):
        """Area-light table f32[L, 16] and total power (nan_ctx_set_area_lights layout)."""
        self._lights = np.ascontiguousarray(lights, dtype=np.float32).reshape(-1, 16)
        lib().oracle_scene_set_area_lights(self.handle, _p(self._lights), self._lights.shape[0], float(power))

    def trace_points(self, lighting, points, iteration, samples, max_bounces, flags=0, precision=F32, threads=0):
        """Irradiance at surface points f32[N, 4] (b1, b2, instance bits,
        primitive bits | back << 31); returns f32[N, 4] and the ray counts."""
        pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 4)
        out = np.zeros_like(pts)
        counts = OracleRayCounts()
        L = lighting_struct(lighting)
        rc = lib().oracle_trace_points(self.handle, ctypes.byref(L), _p(pts), pts.shape[0], iteration, samples,
                                       max_bounces, flags, _p(out), precision, threads, ctypes.byref(counts))
        if rc != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return out, counts.as_dict()

    def trace_probes(self, lighting, values, sample_counts, self_hits, radial, probes,
                     probe_instances, units, iteration, samples_per_probe, max_bounces,
                     reset, precision=F32, threads=0, independent_samples=False):
        """Updates values/sample_counts/self_hits/radial in place."""
        for buf in (values, sample_counts, self_hits, radial):
            assert buf.flags["C_CONTIGUOUS"]
        pr = np.ascontiguousarray(probes).view(np.uint8).reshape(-1)
        pi = np.ascontiguousarray(probe_instances).view(np.uint8).reshape(-1)
        un = np.ascontiguousarray(units, dtype=np.uint32).reshape(-1)
        counts = OracleRayCounts()
        L = lighting_struct(lighting)
        fn = lib().oracle_trace_probes_independent if independent_samples else lib().oracle_trace_probes
        rc = fn(self.handle, ctypes.byref(L), _p(values),
                                       _p(sample_counts), _p(self_hits), _p(radial), _p(pr),
                                       pr.size // 48, _p(pi), pi.size // 48, _p(un), un.size,
                                       iteration, samples_per_probe, max_bounces,
                                       int(bool(reset)), precision, threads,
                                       ctypes.byref(counts))
        if rc != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return counts.as_dict()
