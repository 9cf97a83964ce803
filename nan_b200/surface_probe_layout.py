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

Site placement itself (weighted sample elimination, deficit repair, support
estimation) is the reference's CPU pre-pass; from_sites takes any sites,
e.g. scenes.surface_sites, and the kernel radius follows the reference's
rule max(2.5 * sqrt(area / sites) per instance, 2.5 * sqrt(total area /
total sites), 1e-5).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .surface_probe_octree import build_point_octree, query_probe_indices
from .surface_probe_resources import (SURFACE_PROBE_DTYPE, SURFACE_PROBE_INSTANCE_DTYPE,
                                      SURFACE_PROBE_INSTANCE_SHIFT)


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
                   max_density_multiplier: float = 8.0) -> "SurfaceProbeSiteLayout":
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
        for i in range(n_inst):
            rec = probes[instance_of == i].copy()
            sites = int(fronts[i])
            kernel = max(global_kernel, math.sqrt(areas[i] / sites) * kernel_radius_scale if sites else 0.0, 1e-5)
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
    def build(cls, scene_node, site_count: int, *, seed: int = 1, **kwargs) -> "SurfaceProbeSiteLayout":
        """Area-weighted random sites (scenes.surface_sites) packed by from_sites."""
        from .scenes import surface_sites

        probes, _ = surface_sites(scene_node, site_count, seed=seed)
        return cls.from_sites(scene_node, probes, **kwargs)

    def query_probe_indices(self, instance_index: int, position, radius: float | None = None, normal=None):
        return query_probe_indices(self, instance_index, position, radius, normal)
