"""Surface-probe site layout: per-instance point octrees over given sites,
packed as the reference's SurfaceProbeLayout packs them
(surface_probes.py:2636-2950): per instance the sites' probe records (front,
and a back record with the negated normal for double-sided materials) are
reordered by the instance's point octree, branch child bases and leaf probe
starts are offset into the global arrays, and the instance record holds
(root centre, extent), (node offset, node count, probe offset, probe count)
and (kernel radius, normal cosine threshold, plane sigma = kernel / 4,
triangle-map offset bits). The triangle -> vertex-anchor map has two
records (front, back) per triangle; without anchors every record is
invalid (w = 0).

Sites: build_wse places them as the reference's layout build does before
its repair stages (surface_probes.py:1536-2030): the site budget is split
over instances by area (_allocate_counts, surface_probes.py:265-293), each
instance draws oversample x its count area-weighted candidates
(_sample_instance_surface, :445-497) and weighted sample elimination on the
GPU (all instances in one call, SurfaceProbeSampler) keeps its count.
from_sites takes any sites (e.g. scenes.surface_sites). The kernel radius
follows the reference's rule max(2.5 * sqrt(area / sites), 2.5 * Poisson
radius, 2.5 * sqrt(total area / total sites), 1e-5). Deficit repair, the
protected closure and support estimation are not applied (support 1).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .surface_probe_octree import build_point_octree, query_probe_indices
from .surface_probe_resources import (SURFACE_PROBE_DTYPE, SURFACE_PROBE_INSTANCE_DTYPE,
                                      SURFACE_PROBE_INSTANCE_SHIFT)


def allocate_counts(weights, total: int, *, minimum_per_entry: int = 1) -> np.ndarray:
    """Largest-remainder split of `total` by `weights` with a floor per entry
    (_allocate_counts, surface_probes.py:265-293)."""
    w = np.asarray(weights, dtype=np.float64)
    n = int(w.shape[0])
    if n == 0:
        return np.zeros(0, np.int64)
    floor_each = max(1, int(minimum_per_entry))
    if int(total) < n * floor_each:
        raise ValueError(f"Surface probe budget {total} is smaller than the required {floor_each} samples for "
                         f"each of {n} entries")
    out = np.full(n, floor_each, np.int64)
    rest = int(total) - n * floor_each
    if rest == 0:
        return out
    expected = w / max(float(np.sum(w)), 1e-30) * float(rest)
    extra = np.floor(expected).astype(np.int64)
    out += extra
    left = rest - int(np.sum(extra))
    if left > 0:
        out[np.argsort(-(expected - extra), kind="stable")[:left]] += 1
    return out


@dataclass(frozen=True)
class SurfaceProbeSiteInstance:
    root_center: tuple[float, float, float]
    root_extent: float
    node_offset: int
    node_count: int
    probe_offset: int
    probe_count: int
    kernel_radius: float
    normal_cosine_threshold: float
    plane_sigma: float
    surface_area: float
    surface_site_count: int
    reconstruction_probe_count: int


@dataclass(frozen=True)
class SurfaceProbeSiteLayout:
    probes: np.ndarray
    nodes: np.ndarray
    triangle_vertex_probes: np.ndarray
    instance_gpu_data: np.ndarray
    instance_infos: tuple
    total_probe_count: int
    max_density_multiplier: float

    @classmethod
    def from_sites(cls, scene_node, probes, *, leaf_capacity: int = 8, max_depth: int = 16,
                   kernel_radius_scale: float = 2.5, normal_angle_degrees: float = 45.0,
                   max_density_multiplier: float = 8.0, poisson_radii=None) -> "SurfaceProbeSiteLayout":
        probes = np.asarray(probes, dtype=SURFACE_PROBE_DTYPE)
        instance_of = probes["meta"][:, 3] >> SURFACE_PROBE_INSTANCE_SHIFT
        n_inst = len(scene_node.instances)
        if probes.shape[0] and int(instance_of.max()) >= n_inst:
            raise ValueError("a probe names an instance the scene does not have")
        areas = np.zeros(n_inst)
        tri_counts = np.zeros(n_inst, np.int64)
        for i, (mesh_id, _, transform_id) in enumerate(scene_node.instances):
            mesh = scene_node.meshes[mesh_id]
            m = scene_node.transforms[transform_id].astype(np.float64)
            p = mesh.vertices[:, :3].astype(np.float64) @ m[:3, :3].T + m[:3, 3]
            t = p[mesh.indices.astype(np.int64).reshape(-1, 3)]
            areas[i] = 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1).sum()
            tri_counts[i] = t.shape[0]
        fronts = np.bincount(instance_of[(probes["meta"][:, 3] & 1) == 0], minlength=n_inst)
        total_sites = max(int(fronts.sum()), 1)
        global_kernel = max(math.sqrt(max(float(areas.sum()), 1e-20) / total_sites) * kernel_radius_scale, 1e-5)
        normal_cos = math.cos(math.radians(normal_angle_degrees))

        gpu = np.zeros(n_inst, dtype=SURFACE_PROBE_INSTANCE_DTYPE)
        out_probes, out_nodes, out_maps, infos = [], [], [], []
        node_offset = probe_offset = map_offset = 0
        by_instance = np.argsort(instance_of, kind="stable")
        bounds = np.searchsorted(instance_of[by_instance], np.arange(n_inst + 1))
        for i in range(n_inst):
            rec = probes[by_instance[bounds[i]:bounds[i + 1]]].copy()
            sites = int(fronts[i])
            kernel = max(global_kernel, math.sqrt(areas[i] / sites) * kernel_radius_scale if sites else 0.0,
                         float(poisson_radii[i]) * kernel_radius_scale if poisson_radii is not None else 0.0, 1e-5)
            maps = np.full((int(tri_counts[i]) * 2, 4), 0xFFFFFFFF, np.uint32)
            maps[:, 3] = 0
            if rec.shape[0]:
                rec["position_radius"][:, 3] = kernel
                nodes, order, center, extent = build_point_octree(rec["position_radius"][:, :3],
                                                                  leaf_capacity=leaf_capacity, max_depth=max_depth)
                rec = rec[order]
                nodes = nodes.copy()
                branch = nodes[:, 1] != 0
                nodes[branch, 0] += np.uint32(node_offset)
                nodes[~branch, 2] += np.uint32(probe_offset)
            else:
                nodes = np.zeros((0, 4), np.uint32)
                center, extent = (0.0, 0.0, 0.0), 0.0
            plane_sigma = max(kernel * 0.25, 1e-6)
            gpu["root_center_extent"][i] = (*center, extent)
            gpu["offsets"][i] = (node_offset, nodes.shape[0], probe_offset, rec.shape[0])
            gpu["params"][i] = (kernel, normal_cos, plane_sigma,
                                np.asarray(map_offset, dtype=np.uint32).view(np.float32).item())
            infos.append(SurfaceProbeSiteInstance(center, extent, node_offset, int(nodes.shape[0]), probe_offset,
                                                  int(rec.shape[0]), kernel, normal_cos, plane_sigma,
                                                  float(areas[i]), sites, int(rec.shape[0])))
            out_probes.append(rec)
            out_nodes.append(nodes)
            out_maps.append(maps)
            node_offset += nodes.shape[0]
            probe_offset += rec.shape[0]
            map_offset += maps.shape[0]
        all_nodes = np.concatenate(out_nodes) if node_offset else np.zeros((1, 4), np.uint32)
        all_maps = np.concatenate(out_maps) if map_offset else np.zeros((2, 4), np.uint32)
        return cls(np.concatenate(out_probes), np.ascontiguousarray(all_nodes, np.uint32),
                   np.ascontiguousarray(all_maps, np.uint32), gpu, tuple(infos), int(probe_offset),
                   float(max_density_multiplier))

    @classmethod
    def build_wse(cls, scene_node, target_probe_count: int, *, device=None, oversample_factor: int = 5,
                  seed: int = 1, minimum_per_instance: int = 4, sampler=None, profile: dict | None = None,
                  **kwargs) -> "SurfaceProbeSiteLayout":
        """Sites by weighted sample elimination of oversampled candidates."""
        import time

        from .surface_probe_sampler import SurfaceProbeSampler

        t0 = time.perf_counter()
        tris, areas, double_sided = [], [], []
        for mesh_id, mat_id, transform_id in scene_node.instances:
            mesh = scene_node.meshes[mesh_id]
            m = scene_node.transforms[transform_id].astype(np.float64)
            p = mesh.vertices[:, :3].astype(np.float64) @ m[:3, :3].T + m[:3, 3]
            t = p[mesh.indices.astype(np.int64).reshape(-1, 3)].astype(np.float32)
            tris.append(t)
            e = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]).astype(np.float64)
            areas.append(0.5 * np.linalg.norm(e, axis=1))
            double_sided.append(bool(scene_node.materials[mat_id].double_sided))
        totals = np.array([a.sum() for a in areas])
        counts = allocate_counts(totals, int(target_probe_count),
                                 minimum_per_entry=min(minimum_per_instance,
                                                       max(1, int(target_probe_count) // max(len(totals), 1))))
        cand_pos, cand_nrm, cand_tri, cand_bary, offsets = [], [], [], [], [0]
        for i, (t, a) in enumerate(zip(tris, areas)):
            k = int(counts[i]) * max(1, int(oversample_factor))
            rng = np.random.default_rng([int(seed), i])
            cdf = np.cumsum(a, dtype=np.float64)
            cdf /= cdf[-1]
            cdf[-1] = 1.0
            choice = np.minimum(np.searchsorted(cdf, rng.random(k), side="right"), t.shape[0] - 1)
            uv = rng.random((k, 2), dtype=np.float32)
            su = np.sqrt(uv[:, 0])
            b1 = su * (1.0 - uv[:, 1])
            b2 = su * uv[:, 1]
            ea = t[choice, 1] - t[choice, 0]
            eb = t[choice, 2] - t[choice, 0]
            cand_pos.append((t[choice, 0] + ea * b1[:, None] + eb * b2[:, None]).astype(np.float32))
            cr = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]).astype(np.float64)
            fn = cr / np.maximum(np.linalg.norm(cr, axis=1, keepdims=True), 1e-30)
            cand_nrm.append(fn[choice].astype(np.float32))
            cand_tri.append(choice.astype(np.uint32))
            cand_bary.append(np.stack((b1, b2), axis=1).astype(np.float32))
            offsets.append(offsets[-1] + k)
        t1 = time.perf_counter()
        if sampler is None:
            from .scene import Device

            sampler = SurfaceProbeSampler(device if device is not None else Device(0))
        keep, radii = sampler.eliminate(np.concatenate(cand_pos), np.concatenate(cand_nrm), offsets, counts, totals)
        keep = keep.cpu().numpy().astype(bool)
        t2 = time.perf_counter()
        records = []
        for i in range(len(tris)):
            sel = np.flatnonzero(keep[offsets[i]:offsets[i + 1]])
            pos = cand_pos[i][sel]
            for side in range(2 if double_sided[i] else 1):
                r = np.zeros(sel.shape[0], dtype=SURFACE_PROBE_DTYPE)
                r["position_radius"][:, :3] = pos
                r["normal_side"][:, :3] = cand_nrm[i][sel] * (-1.0 if side else 1.0)
                r["normal_side"][:, 3] = 1.0
                r["meta"][:, 0] = cand_tri[i][sel]
                r["meta"][:, 1] = cand_bary[i][sel, 0].view(np.uint32)
                r["meta"][:, 2] = cand_bary[i][sel, 1].view(np.uint32)
                r["meta"][:, 3] = (1 if side else 0) | (i << SURFACE_PROBE_INSTANCE_SHIFT)
                records.append(r)
        layout = cls.from_sites(scene_node, np.concatenate(records), poisson_radii=radii, **kwargs)
        if profile is not None:
            profile.update(candidates_s=t1 - t0, elimination_s=t2 - t1, packing_s=time.perf_counter() - t2,
                           candidates=int(offsets[-1]), rounds=int(sampler.last_rounds))
        return layout

    @classmethod
    def build(cls, scene_node, site_count: int, *, seed: int = 1, **kwargs) -> "SurfaceProbeSiteLayout":
        """Area-weighted random sites (scenes.surface_sites) packed by from_sites."""
        from .scenes import surface_sites

        probes, _ = surface_sites(scene_node, site_count, seed=seed)
        return cls.from_sites(scene_node, probes, **kwargs)

    def query_probe_indices(self, instance_index: int, position, radius: float | None = None, normal=None):
        return query_probe_indices(self, instance_index, position, radius, normal)
