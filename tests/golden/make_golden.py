"""Generate golden input/output vectors from the reference's own Python code.

Run where the reference project is checked out (default: a ``reference``
folder beside this repository's folder; override with
``NAN_REFERENCE_ROOT``)::

    python tests/golden/make_golden.py

It imports the reference's numpy reference functions -- the RGB9E5 pack/unpack
of ``test_mesh_colors_rgb9e5.py:15-50``, the hemi-oct encode/decode of
``surface_probes.py:45-110``, the Mesh Colors lattice math of
``mesh_colors.py:24-79``, the FP64 brute-force any-hit caster of
``vertex_baker/visibility_baker.py:348-402``, the point octree builder and
query of ``surface_probes.py:1348-1438, 3007-3099``, the Python weighted
sample elimination of ``surface_probes.py:897-985``, and the Python deficit
repair and support estimate of ``surface_probe_sampler.py:990-1103,
1179-1260`` -- with the graphics-only modules
(slangpy, trimesh, pygltflib, PIL) replaced by inert stand-ins, evaluates them
on seeded inputs, and writes ``reference_vectors.npz`` next to this file.
The GPU box never runs this script; tests read the committed ``.npz`` only.
"""

from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("NAN_REFERENCE_ROOT", HERE.parents[2] / "reference"))


class _InertMeta(type):
    """Class-level attribute lookups of a stub (``spy.KeyCode.a``) yield inert values too."""

    def __getattr__(cls, name):
        return _Inert()


class _Inert(metaclass=_InertMeta):
    """Stand-in for any attribute of a stubbed graphics module."""

    def __init__(self, *args, **kwargs):
        pass

    def __call__(self, *args, **kwargs):
        return _Inert()

    def __getattr__(self, name):
        return _Inert()


def _stub(name: str) -> None:
    module = types.ModuleType(name)
    module.__getattr__ = lambda attr: _Inert  # type: ignore[attr-defined]
    sys.modules[name] = module


def _install_stubs() -> None:
    for name in ("slangpy", "slangpy.math", "trimesh", "pygltflib", "PIL",
                 "PIL.Image", "OpenEXR", "event_dispatching"):
        _stub(name)
    sys.modules["slangpy"].math = sys.modules["slangpy.math"]  # type: ignore[attr-defined]
    scene_node = types.ModuleType("scene_node")
    scene_node.SceneNode = _Inert  # type: ignore[attr-defined]
    sys.modules["scene_node"] = scene_node


class _F32(np.ndarray):
    """float32 vector standing in for slangpy's float2/float3 (components .x/.y/.z)."""

    x = property(lambda self: self[0])
    y = property(lambda self: self[1])
    z = property(lambda self: self[2])


def _f32(*components):
    return np.asarray(components, dtype=np.float32).view(_F32)


def _host_records(out: dict) -> None:
    """Host-side records of the reference's own Python: the Halton jitter of
    Camera.begin_frame (camera.py:4-23, 87-96), the mesh factories
    (mesh.py:31-189) and the 16-byte descriptor packing (scene.py:85-108).
    slangpy's float2 and frac are stood in by float32 numpy arrays; the
    camera's image-plane basis and the transform matrices go through slangpy
    math that is not installed here, so they are not recorded."""
    for name in ("event_dispatcher", "event_dispatcher.sync_dispatcher"):
        _stub(name)
    import camera as ref_camera  # noqa: E402
    import mesh as ref_mesh  # noqa: E402
    import scene as ref_scene  # noqa: E402

    spy = sys.modules["slangpy"]
    spy.float2 = _f32
    spy.math.frac = lambda v: (v - np.floor(v)).astype(np.float32).view(_F32)
    out["halton_index"] = np.arange(0, 200, dtype=np.int64)
    out["halton_base2"] = np.asarray([ref_camera.halton(i, 2) for i in range(200)], np.float64)
    out["halton_base3"] = np.asarray([ref_camera.halton(i, 3) for i in range(200)], np.float64)
    sizes = np.asarray([[256, 256], [1920, 1080], [3840, 2160], [64, 48]], np.int64)
    jitter = np.zeros((sizes.shape[0], 40, 2), np.float32)
    for k, (w, h) in enumerate(sizes):
        cam = object.__new__(ref_camera.Camera)  # begin_frame's own code, without the slangpy basis
        cam.sample_pattern = ref_camera.HaltonSamplePattern(16)
        cam.jitter = _f32(0.0, 0.0)
        cam.frame_index = 0
        cam._has_prev_matrices = False
        cam.recompute = lambda: None
        for f in range(40):
            cam.begin_frame(int(w), int(h))
            jitter[k, f] = (cam.jitter.x, cam.jitter.y)
    out["camera_sizes"] = sizes
    out["camera_jitter"] = jitter

    meshes = {
        "cube_1": ref_mesh.Mesh.create_cube((1.0, 1.0, 1.0)),
        "cube_a": ref_mesh.Mesh.create_cube((0.6, 1.2, 0.6)),
        "cube_b": ref_mesh.Mesh.create_cube((2.5, 0.3, 1.1)),
        "quad": ref_mesh.Mesh.create_quad((2.0, 3.0)),
        "quad_yz_pos": ref_mesh.Mesh.create_quad_yz((2.0, 3.0), True),
        "quad_yz_neg": ref_mesh.Mesh.create_quad_yz((2.0, 3.0), False),
        "quad_xy_pos": ref_mesh.Mesh.create_quad_xy((2.0, 3.0), True),
        "quad_xy_neg": ref_mesh.Mesh.create_quad_xy((2.0, 3.0), False),
    }
    for key, m in meshes.items():
        out[f"mesh_{key}_vertices"] = np.asarray(m.vertices, np.float32)
        out[f"mesh_{key}_indices"] = np.asarray(m.indices, np.uint32)
    mesh_fields = np.asarray([[36, 108, 0, 0], [24, 36, 36, 108], [4, 6, 60, 144]], np.uint32)
    inst_fields = np.asarray([[0, 1, 0, 0], [2, 0, 5, 1], [1, 3, 2, 0]], np.uint32)
    out["desc_mesh_fields"] = mesh_fields
    out["desc_mesh_packed"] = np.frombuffer(
        b"".join(ref_scene.Scene.MeshDesc(*map(int, r)).pack() for r in mesh_fields), np.uint32).reshape(-1, 4)
    out["desc_instance_fields"] = inst_fields
    out["desc_instance_packed"] = np.frombuffer(
        b"".join(ref_scene.Scene.InstanceDesc(*map(int, r)).pack() for r in inst_fields), np.uint32).reshape(-1, 4)


def main() -> None:
    _install_stubs()
    sys.path.insert(0, str(REF))
    sys.path.insert(0, str(REF / "vertex_baker"))

    import mesh_colors  # noqa: E402
    import surface_probes  # noqa: E402
    import test_mesh_colors_rgb9e5 as rgb9e5_test  # noqa: E402
    import visibility_baker  # noqa: E402

    rng = np.random.default_rng(20261203)
    out: dict[str, np.ndarray] = {}

    # RGB9E5: the reference test's seven values first, then seeded values
    # spread over the representable exponent range (plus clamped extremes).
    golden = np.asarray(
        [
            [0.0, 0.0, 0.0],
            [1.0, 1.0, 1.0],
            [0.25, 0.5, 1.0],
            [100.0, 10.0, 1.0],
            [65408.0, 65408.0, 65408.0],
            [-1.0, np.nan, np.inf],
            [2.0**-24, 2.0**-20, 2.0**-16],
        ],
        dtype=np.float32,
    )
    magnitudes = np.exp2(rng.uniform(-28.0, 17.0, size=(4000, 1)))
    randoms = (rng.uniform(0.0, 1.0, size=(4000, 3)) * magnitudes).astype(np.float32)
    values = np.concatenate([golden, randoms], axis=0)
    packed = np.asarray(
        [rgb9e5_test._pack_rgb9e5_reference(v) for v in values], dtype=np.uint32
    )
    decoded = np.stack([rgb9e5_test._unpack_rgb9e5_reference(p) for p in packed])
    out["rgb9e5_values"] = values
    out["rgb9e5_packed"] = packed
    out["rgb9e5_decoded"] = decoded.astype(np.float32)

    # Hemi-oct: canonical directions of test_surface_probes.py:95-116, then a
    # seeded hemisphere set as in its round-trip test.
    canonical = np.asarray(
        [[0, 0, 1], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0]], dtype=np.float32
    )
    dirs = rng.normal(size=(4096, 3)).astype(np.float32)
    dirs[:, 2] = np.abs(dirs[:, 2])
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    dirs = np.concatenate([canonical, dirs], axis=0).astype(np.float32)
    uv = surface_probes.surface_probe_hemi_oct_encode(dirs)
    out["hemi_dirs"] = dirs
    out["hemi_uv"] = uv.astype(np.float32)
    out["hemi_decoded"] = surface_probes.surface_probe_hemi_oct_decode(uv).astype(np.float32)

    # Mesh Colors lattice addressing.
    addr, res, ij = [], [], []
    for resolution in (1, 2, 4, 8, 16, 32, 64):
        for address in range(mesh_colors.colors_per_patch(resolution)):
            i, j = mesh_colors.address_to_ij(address, resolution)
            assert mesh_colors.ij_to_address(i, j, resolution) == address
            addr.append(address)
            res.append(resolution)
            ij.append((i, j))
    out["mc_address"] = np.asarray(addr, dtype=np.uint32)
    out["mc_resolution"] = np.asarray(res, dtype=np.uint32)
    out["mc_ij"] = np.asarray(ij, dtype=np.uint32)

    # Any-hit visibility against a seeded triangle soup with the reference's
    # FP64 Moller-Trumbore brute force.
    tris = rng.uniform(-1.0, 1.0, size=(64, 3, 3)).astype(np.float32)
    origins = rng.uniform(-1.5, 1.5, size=(2048, 3)).astype(np.float32)
    directions = rng.normal(size=(2048, 3)).astype(np.float32)
    directions /= np.linalg.norm(directions, axis=1, keepdims=True)
    directions = directions.astype(np.float32)
    occluded = visibility_baker._intersects_any_bruteforce(
        origins, directions, tris, max_distance=1.25, ray_epsilon=1e-6
    )
    out["vis_triangles"] = tris
    out["vis_origins"] = origins
    out["vis_directions"] = directions
    out["vis_max_distance"] = np.asarray([1.25], dtype=np.float32)
    out["vis_occluded"] = occluded.astype(np.uint8)

    # Point octree: the two cases of test_surface_probes.py:133-190 (boundary
    # points on the float32 centre; a degenerate single-octant chain), and
    # clustered sites on two facing sheets with the layout defaults, plus
    # radius queries with and without the normal gate on the last one. Each
    # case has its own generator so the vectors above stay as they were.
    cases = []
    a = np.random.default_rng(1234).uniform(-2.0, 3.0, size=(4097, 3)).astype(np.float32)
    a[:8] = np.array([[0.5, 0.5, 0.5], [0.5, 0.5, -2.0], [0.5, -2.0, 0.5], [0.5, -2.0, -2.0],
                      [-2.0, 0.5, 0.5], [-2.0, 0.5, -2.0], [-2.0, -2.0, 0.5], [-2.0, -2.0, -2.0]], np.float32)
    cases.append((a, 8, 12))
    cases.append((np.zeros((33, 3), np.float32), 1, 5))
    crng = np.random.default_rng(77)
    sheet = crng.uniform(0.0, 4.0, size=(3000, 2))
    c = np.zeros((6000, 3), np.float32)
    c[:3000, 0], c[:3000, 2] = sheet[:, 0], sheet[:, 1]
    c[3000:, 0], c[3000:, 2] = sheet[:, 0], sheet[:, 1]
    c[3000:, 1] = 0.05
    c[100:140] = c[99]  # exact duplicates fill one leaf past capacity
    cases.append((c, 8, 16))
    for k, (pos, leaf, depth) in enumerate(cases):
        nodes, order, center, extent = surface_probes._build_point_octree_python(
            pos, leaf_capacity=leaf, max_depth=depth)
        out[f"octree{k}_positions"] = pos
        out[f"octree{k}_params"] = np.asarray([leaf, depth], np.uint32)
        out[f"octree{k}_nodes"] = np.asarray(nodes, np.uint32)
        out[f"octree{k}_order"] = np.asarray(order, np.int64)
        out[f"octree{k}_root"] = np.asarray([*center, extent], np.float64)
    pos = cases[2][0]
    nodes, order, center, extent = surface_probes._build_point_octree_python(pos, leaf_capacity=8, max_depth=16)
    probes = np.zeros(pos.shape[0], dtype=surface_probes.SURFACE_PROBE_DTYPE)
    probes["position_radius"][:, :3] = pos[order]
    normals = np.zeros((pos.shape[0], 3), np.float32)
    normals[:3000, 1] = 1.0
    normals[3000:, 1] = -1.0
    probes["normal_side"][:, :3] = normals[order]
    info = types.SimpleNamespace(node_offset=0, root_center=center, root_extent=extent, kernel_radius=0.3)
    layout = types.SimpleNamespace(instance_infos=[info], nodes=nodes, probes=probes,
                                   _sphere_intersects_cube=surface_probes.SurfaceProbeLayout._sphere_intersects_cube)
    qrng = np.random.default_rng(91)
    queries = np.concatenate([qrng.uniform(-0.2, 4.2, size=(200, 1)), qrng.uniform(-0.1, 0.15, size=(200, 1)),
                              qrng.uniform(-0.2, 4.2, size=(200, 1))], axis=1)
    radii = qrng.uniform(0.0, 0.6, size=200)
    found, offsets, qnormals = [], [0], []
    for i in range(200):
        qn = None if i % 2 == 0 else (0.0, 1.0 if i % 4 == 1 else -1.0, 0.0)
        r = None if i % 10 == 3 else float(radii[i])
        idx = surface_probes.SurfaceProbeLayout.query_probe_indices(layout, 0, queries[i], radius=r, normal=qn)
        found.append(np.asarray(idx, np.int64))
        offsets.append(offsets[-1] + len(idx))
        qnormals.append((0.0, 0.0, 0.0) if qn is None else qn)
    out["octree_query_positions"] = queries
    out["octree_query_radii"] = np.where(np.arange(200) % 10 == 3, -1.0, radii)
    out["octree_query_normals"] = np.asarray(qnormals, np.float64)
    out["octree_query_found"] = np.concatenate(found)
    out["octree_query_offsets"] = np.asarray(offsets, np.int64)

    # Weighted sample elimination (the reference's Python backend): random
    # candidates on a plane, on two facing sheets plus a wall, and the
    # regular grid of test_surface_probes.py:194-230.
    wrng = np.random.default_rng(4242)
    wse_cases = []
    p = np.zeros((2000, 3), np.float32)
    p[:, 0], p[:, 2] = wrng.uniform(0.0, 1.0, 2000), wrng.uniform(0.0, 1.0, 2000)
    n = np.tile(np.float32([0.0, 1.0, 0.0]), (2000, 1))
    wse_cases.append((p, n, 400, 1.0))
    m = 3000
    p = np.zeros((m, 3), np.float32)
    n = np.zeros((m, 3), np.float32)
    u = wrng.uniform(0.0, 1.0, (m, 2)).astype(np.float32)
    p[:1000, 0], p[:1000, 2], n[:1000, 1] = u[:1000, 0], u[:1000, 1], 1.0
    p[1000:2000, 0], p[1000:2000, 2], p[1000:2000, 1], n[1000:2000, 1] = u[1000:2000, 0], u[1000:2000, 1], 0.05, -1.0
    p[2000:, 1], p[2000:, 2], n[2000:, 0] = u[2000:, 0], u[2000:, 1], 1.0
    wse_cases.append((p, n, 600, 3.0))
    c = np.linspace(0.0, 1.0, 20, dtype=np.float32)
    gx, gz = np.meshgrid(c, c, indexing="xy")
    p = np.stack((gx.reshape(-1), np.zeros(gx.size, np.float32), gz.reshape(-1)), axis=1).astype(np.float32)
    n = np.tile(np.float32([0.0, 1.0, 0.0]), (p.shape[0], 1))
    wse_cases.append((p, n, 64, 1.0))
    for k, (pos, nrm, count, area) in enumerate(wse_cases):
        sel, radius = surface_probes._weighted_sample_elimination_python(pos, nrm, count, surface_area=area)
        out[f"wse{k}_positions"] = pos
        out[f"wse{k}_normals"] = nrm
        out[f"wse{k}_params"] = np.asarray([count, area], np.float64)
        out[f"wse{k}_selected"] = np.asarray(sel, np.int64)
        out[f"wse{k}_radius"] = np.asarray([radius], np.float64)

    # Deficit repair (the reference's Python form): the cases of
    # test_surface_probes.py:436-600 and a seeded two-instance case.
    import surface_probe_sampler

    up = np.float32([0.0, 1.0, 0.0])
    rep_cases = []
    bp = np.float32([[0, 0, 0], [1, 0, 0]])
    cp = np.float32([[0.1, 0, 0], [0.2, 0, 0], [0.9, 0, 0]])
    rep_cases.append((bp, np.tile(up, (2, 1)), np.zeros(2, np.uint32), cp, np.tile(up, (3, 1)),
                      np.zeros(3, np.uint32), bp.copy(), np.tile(up, (2, 1)), np.zeros(2, np.uint32),
                      np.float32([0.5]), 3, 3))
    bp = np.float32([[9.9, 0, 0], [10.0, 0, 0], [10.1, 0, 0]])
    cp = np.float32([[0.0, 0, 0], [0.02, 0, 0], [0.04, 0, 0], [0.06, 0, 0], [0.08, 0, 0], [10.2, 0, 0]])
    rep_cases.append((bp, np.tile(up, (3, 1)), np.zeros(3, np.uint32), cp, np.tile(up, (6, 1)),
                      np.zeros(6, np.uint32), np.float32([[0, 0, 0], [10, 0, 0]]), np.tile(up, (2, 1)),
                      np.zeros(2, np.uint32), np.float32([0.5]), 4, 6))
    rrng = np.random.default_rng(31)

    def sheet(n, inst, normal, offset):
        p = np.zeros((n, 3), np.float32)
        u = rrng.uniform(0.0, 2.0, (n, 2)).astype(np.float32)
        if normal[1] != 0:
            p[:, 0], p[:, 2], p[:, 1] = u[:, 0], u[:, 1], offset
        else:
            p[:, 1], p[:, 2], p[:, 0] = u[:, 0], u[:, 1], offset
        return p, np.tile(np.float32(normal), (n, 1)), np.full(n, inst, np.uint32)

    b0, b1 = sheet(60, 0, [0, 1, 0], 0.0), sheet(25, 1, [1, 0, 0], 3.0)
    c0, c1 = sheet(400, 0, [0, 1, 0], 0.0), sheet(300, 1, [1, 0, 0], 3.0)
    a0, a1 = sheet(500, 0, [0, 1, 0], 0.0), sheet(400, 1, [1, 0, 0], 3.0)
    cat = lambda x, y: tuple(np.concatenate([x[k], y[k]]) for k in range(3))
    rep_cases.append((*cat(b0, b1), *cat(c0, c1), *cat(a0, a1), np.float32([0.35, 0.5]), 4, 120))
    for k, (bp, bn, bi, cp, cn, ci, ap, an, ai, radii, mg, budget) in enumerate(rep_cases):
        res = surface_probe_sampler.deficit_repair_python(bp, bn, bi, cp, cn, ci, ap, an, ai, radii,
                                                          min_gather_count=mg, max_repair_count=budget,
                                                          normal_cosine_threshold=0.5)
        for name, value in (("bp", bp), ("bn", bn), ("bi", bi), ("cp", cp), ("cn", cn), ("ci", ci), ("ap", ap),
                            ("an", an), ("ai", ai), ("radii", radii)):
            out[f"rep{k}_{name}"] = np.asarray(value)
        out[f"rep{k}_params"] = np.asarray([mg, budget], np.uint32)
        out[f"rep{k}_selected"] = np.asarray(res.selected_candidate_indices, np.int64)
        for name in ("counts_before", "counts_after", "weight_sums_before", "weight_sums_after", "ess_before",
                     "ess_after"):
            out[f"rep{k}_{name}"] = np.asarray(getattr(res, name))

    # Support estimate (the reference's Python form): two instances, one a
    # tilted sheet so the plane and normal terms are not axis aligned, and
    # query sites in the interior and at the borders.
    srng = np.random.default_rng(57)
    nrm1 = np.float32([0.3, 0.9, 0.2])
    nrm1 /= np.linalg.norm(nrm1)
    t1 = np.cross(nrm1, [1.0, 0.0, 0.0])
    t1 /= np.linalg.norm(t1)
    b1 = np.cross(nrm1, t1)
    u = srng.uniform(0.0, 3.0, (2500, 2))
    ref1 = (5.0 + u[:, :1] * t1 + u[:, 1:] * b1).astype(np.float32)
    ref0 = np.zeros((2000, 3), np.float32)
    ref0[:, 0], ref0[:, 2] = srng.uniform(0, 2, 2000), srng.uniform(0, 2, 2000)
    rp = np.concatenate([ref0, ref1])
    rn = np.concatenate([np.tile(np.float32([0, 1, 0]), (2000, 1)), np.tile(nrm1.astype(np.float32), (2500, 1))])
    ri = np.concatenate([np.zeros(2000, np.uint32), np.ones(2500, np.uint32)])
    ra = np.concatenate([np.full(2000, 4.0 / 2000, np.float32), np.full(2500, 9.0 / 2500, np.float32)])
    qp = np.concatenate([ref0[:150], ref1[:150]]).copy()
    qn = np.concatenate([rn[:150], rn[2000:2150]])
    qi = np.concatenate([np.zeros(150, np.uint32), np.ones(150, np.uint32)])
    radii = np.float32([0.12, 0.2])
    res = surface_probe_sampler.estimate_support_python(rp, rn, ri, ra, qp, qn, qi, radii, normal_cosine_threshold=0.5)
    for name, value in (("rp", rp), ("rn", rn), ("ri", ri), ("ra", ra), ("qp", qp), ("qn", qn), ("qi", qi),
                        ("radii", radii), ("f", res.support_f), ("m", res.density_m)):
        out[f"sup_{name}"] = np.asarray(value)
    # a dense case: 30000 reference points, radius 0.6, so each query sums
    # 10^4 to 2.5 x 10^4 terms (several of numpy's 8192-element buffers)
    u = srng.uniform(0.0, 1.0, (30000, 2)).astype(np.float32)
    rp = np.stack([u[:, 0], 0.02 * np.sin(7.0 * u[:, 1]), u[:, 1]], axis=1).astype(np.float32)
    rn = np.tile(np.float32([0, 1, 0]), (30000, 1))
    ri = np.zeros(30000, np.uint32)
    ra = (srng.uniform(0.5, 1.5, 30000) / 30000).astype(np.float32)
    qp, qn, qi = rp[:24].copy(), rn[:24].copy(), ri[:24].copy()
    radii = np.float32([0.6])
    res = surface_probe_sampler.estimate_support_python(rp, rn, ri, ra, qp, qn, qi, radii, normal_cosine_threshold=0.5)
    for name, value in (("rp", rp), ("rn", rn), ("ri", ri), ("ra", ra), ("qp", qp), ("qn", qn), ("qi", qi),
                        ("radii", radii), ("f", res.support_f), ("m", res.density_m)):
        out[f"supd_{name}"] = np.asarray(value)

    # Adaptive weighted sample elimination (the reference's Python form):
    # random candidates on a plane with a 4:1 density step and jitter, two
    # facing sheets plus a wall with smoothly varying densities, and the
    # tie-heavy density grid of test_surface_probes.py:312-377.
    arng = np.random.default_rng(77)
    awse_cases = []
    p = np.zeros((2000, 3), np.float32)
    p[:, 0], p[:, 2] = arng.uniform(0.0, 1.0, 2000), arng.uniform(0.0, 1.0, 2000)
    d = (np.where(p[:, 0] < 0.5, 1.6, 0.4) * arng.uniform(0.8, 1.25, 2000)).astype(np.float32)
    awse_cases.append((p, np.tile(np.float32([0.0, 1.0, 0.0]), (2000, 1)), d, 300, 1.0))
    m = 3000
    p = np.zeros((m, 3), np.float32)
    n = np.zeros((m, 3), np.float32)
    u = arng.uniform(0.0, 1.0, (m, 2)).astype(np.float32)
    p[:1000, 0], p[:1000, 2], n[:1000, 1] = u[:1000, 0], u[:1000, 1], 1.0
    p[1000:2000, 0], p[1000:2000, 2], p[1000:2000, 1], n[1000:2000, 1] = u[1000:2000, 0], u[1000:2000, 1], 0.05, -1.0
    p[2000:, 1], p[2000:, 2], n[2000:, 0] = u[2000:, 0], u[2000:, 1], 1.0
    d = (0.5 + 1.5 * u[:, 0] * u[:, 0]).astype(np.float32)
    awse_cases.append((p, n, d, 500, 3.0))
    c = np.linspace(0.0, 1.0, 20, dtype=np.float32)
    gx, gz = np.meshgrid(c, c, indexing="xy")
    p = np.stack((gx.reshape(-1), np.zeros(gx.size, np.float32), gz.reshape(-1)), axis=1).astype(np.float32)
    d = np.where(p[:, 0] < 0.5, 1.6, 0.4).astype(np.float32)
    awse_cases.append((p, np.tile(np.float32([0.0, 1.0, 0.0]), (p.shape[0], 1)), d, 64, 1.0))
    for k, (pos, nrm, dens, count, area) in enumerate(awse_cases):
        sel, radius = surface_probes._adaptive_weighted_sample_elimination_python(pos, nrm, dens, count,
                                                                                  surface_area=area)
        out[f"awse{k}_positions"] = pos
        out[f"awse{k}_normals"] = nrm
        out[f"awse{k}_densities"] = dens
        out[f"awse{k}_params"] = np.asarray([count, area], np.float64)
        out[f"awse{k}_selected"] = np.asarray(sel, np.int64)
        out[f"awse{k}_radius"] = np.asarray([radius], np.float64)

    # Audit/repair candidate filter (the reference's Python form,
    # _deduplicate_audit_candidates and _exclude_selected_duplicates): the
    # case of test_surface_probes.py:697-730 and random candidates whose
    # second half repeats the first, every third base site selected.
    frng = np.random.default_rng(91)
    flt_cases = []
    p = np.float32([[0.0, 0, 0], [0.1, 0, 0], [0.0, 0, 0], [0.2, 0, 0], [1.1, 0, 0]])
    n = np.float32([[0, 1, 0], [0, 1, 0], [0, 1, 0], [0, -1, 0], [0, 1, 0]])
    flt_cases.append((p, n, np.uint32([0]), 1.0))
    p = frng.uniform(-1.0, 1.0, (6000, 3)).astype(np.float32)
    n = frng.normal(size=(6000, 3)).astype(np.float32)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-20)
    p[3000:], n[3000:] = p[:3000], n[:3000]
    flt_cases.append((p, n, np.arange(0, 3000, 3, dtype=np.uint32), 0.05))
    for k, (pos, nrm, sel, cell) in enumerate(flt_cases):
        cands = surface_probes._InstanceCandidates(pos, nrm, np.zeros((pos.shape[0], 2), np.float32),
                                                   np.zeros(pos.shape[0], np.uint32), 1.0)
        audit = surface_probes._deduplicate_audit_candidates(cands, cell, 0.5)
        repair = surface_probes._exclude_selected_duplicates(cands, cands, sel.astype(np.int64))
        # the subsets carry positions; map them back to candidate indices
        index_of = {}
        for i in range(pos.shape[0]):
            index_of.setdefault((pos[i].tobytes(), nrm[i].tobytes()), []).append(i)

        def indices(subset):
            taken = {}
            res = []
            for q in range(subset.positions.shape[0]):
                key = (subset.positions[q].tobytes(), subset.normals[q].tobytes())
                j = taken.get(key, 0)
                res.append(index_of[key][j])
                taken[key] = j + 1
            return np.asarray(res, np.int64)

        out[f"flt{k}_positions"] = pos
        out[f"flt{k}_normals"] = nrm
        out[f"flt{k}_selected_base"] = sel
        out[f"flt{k}_cell"] = np.asarray([cell], np.float64)
        out[f"flt{k}_audit"] = indices(audit)
        out[f"flt{k}_repair"] = indices(repair)

    _host_records(out)
    np.savez_compressed(HERE / "reference_vectors.npz", **out)
    print("wrote", HERE / "reference_vectors.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
