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

Sites: build_wse places them as the reference's layout build does
(surface_probes.py:1536-2420): the site budget is split
over instances by area (_allocate_counts, surface_probes.py:265-293), each
instance draws oversample x its count area-weighted candidates
(_sample_instance_surface, :445-497) and weighted sample elimination on the
GPU (all instances in one call, SurfaceProbeSampler) keeps its count.
from_sites takes any sites (e.g. scenes.surface_sites). The kernel radius
follows the reference's rule max(2.5 * sqrt(area / sites), 2.5 * Poisson
radius, 2.5 * sqrt(total area / total sites), 1e-5), fixed before the
deficit repair adds up to 30 % more sites where audit points gather fewer
than 4 (surface_probes.py:2380-2420), and each site's support f
(estimate_surface_support against the candidate population, area /
candidates each, surface_probes.py:2586-2604) goes into its record. The
protected closure is not applied.
"""

from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass

import numpy as np

from .surface_probe_octree import build_point_octree, query_probe_indices
from .surface_probe_resources import (SURFACE_PROBE_DTYPE, SURFACE_PROBE_FLAG_PROTECTED,
                                      SURFACE_PROBE_FLAG_VERTEX_ANCHOR, SURFACE_PROBE_INSTANCE_DTYPE,
                                      SURFACE_PROBE_INSTANCE_SHIFT)


def allocate_density_counts(weights, density: float, *, minimum_per_entry: int = 1) -> np.ndarray:
    """Site counts from an absolute density (_allocate_density_counts,
    surface_probes.py:296-324): floor(weight x density + 0.5) + the floor
    per entry; the total is an output."""
    w = np.asarray(weights, dtype=np.float64)
    density = float(density)
    if not math.isfinite(density) or density <= 0.0:
        raise ValueError("Surface probe density must be finite and positive")
    return np.floor(w * density + 0.5).astype(np.int64) + np.int64(max(1, int(minimum_per_entry)))


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


def _surface_points(t, areas, k, rng, densities=None):
    """k area-weighted points on triangles t (_sample_instance_surface,
    surface_probes.py:445-497), area x density weighted when densities are
    given: (positions, face normals, triangle, b1, b2)."""
    weights = areas if densities is None else areas * np.asarray(densities, dtype=np.float64)
    cdf = np.cumsum(weights, dtype=np.float64)
    cdf /= cdf[-1]
    cdf[-1] = 1.0
    choice = np.minimum(np.searchsorted(cdf, rng.random(k), side="right"), t.shape[0] - 1)
    uv = rng.random((k, 2), dtype=np.float32)
    su = np.sqrt(uv[:, 0])
    b1 = (su * (1.0 - uv[:, 1])).astype(np.float32)
    b2 = (su * uv[:, 1]).astype(np.float32)
    ea = t[choice, 1] - t[choice, 0]
    eb = t[choice, 2] - t[choice, 0]
    pos = (t[choice, 0] + ea * b1[:, None] + eb * b2[:, None]).astype(np.float32)
    return pos, _face_normals(t)[choice], choice.astype(np.uint32), b1, b2


def _surface_points_group(t, areas, counts, rng, densities=None):
    """_surface_points for the g instances of one mesh at once: t f32[g, T,
    3, 3], areas [g, T], counts[g] points per instance, densities [g, T] or
    None; one random stream for the group. Returns one tuple per instance."""
    cols = _surface_points_group_flat(t, areas, counts, rng, densities)
    parts = np.cumsum(np.asarray(counts, dtype=np.int64))[:-1]
    cols = [np.split(c, parts) for c in cols]
    return [tuple(c[j] for c in cols) for j in range(areas.shape[0])]


def _surface_points_group_flat(t, areas, counts, rng, densities=None, normals=None):
    """_surface_points_group's points back to back, instance by instance:
    (pos, nrm, tri, b1, b2). normals: the triangles' _face_normals [g, T, 3]
    when already known."""
    g, n = areas.shape
    w = areas if densities is None else areas * np.asarray(densities, dtype=np.float64)
    cdf = np.cumsum(w, axis=1, dtype=np.float64)
    cdf /= cdf[:, -1:]
    cdf[:, -1] = 1.0
    counts = np.asarray(counts, dtype=np.int64)
    rows = np.repeat(np.arange(g), counts)
    # row r's distribution shifted to [r, r + 1]: one search for every row
    flat = (cdf + np.arange(g, dtype=np.float64)[:, None]).reshape(-1)
    choice = np.searchsorted(flat, rng.random(rows.size) + rows, side="right") - rows * n
    choice = np.clip(choice, 0, n - 1)
    uv = rng.random((rows.size, 2), dtype=np.float32)
    su = np.sqrt(uv[:, 0])
    b1 = (su * (1.0 - uv[:, 1])).astype(np.float32)
    b2 = (su * uv[:, 1]).astype(np.float32)
    tt = t[rows, choice]
    pos = (tt[:, 0] + (tt[:, 1] - tt[:, 0]) * b1[:, None] + (tt[:, 2] - tt[:, 0]) * b2[:, None]).astype(np.float32)
    nrm = _face_normals(tt) if normals is None else normals[rows, choice]
    return pos, nrm, choice.astype(np.uint32), b1, b2


class _PointSets:
    """Surface points of every instance back to back, instance by instance:
    pos f32[N, 3], nrm f32[N, 3], tri u32[N], b1, b2 f32[N]; instance i's
    points at starts[i]:starts[i + 1]."""

    __slots__ = ("cols", "starts")

    def __init__(self, cols, counts):
        self.cols = tuple(cols)
        self.starts = np.concatenate([[0], np.cumsum(np.asarray(counts, dtype=np.int64))])

    @property
    def n(self) -> int:
        return int(self.starts[-1])

    @property
    def counts(self) -> np.ndarray:
        return np.diff(self.starts)

    @property
    def inst(self) -> np.ndarray:
        return np.repeat(np.arange(self.starts.shape[0] - 1, dtype=np.uint32), self.counts)

    def take(self, idx) -> "_PointSets":
        """The points at ascending global indices idx."""
        idx = np.asarray(idx, dtype=np.int64)
        return _PointSets((c[idx] for c in self.cols), np.diff(np.searchsorted(idx, self.starts)))

    @classmethod
    def from_groups(cls, groups, n_inst: int) -> "_PointSets":
        """Point sets from per-mesh-group outputs -- (members, counts per
        member, columns back to back in member order) -- in instance order."""
        if not groups:
            return cls((np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), np.zeros(0, np.uint32),
                        np.zeros(0, np.float32), np.zeros(0, np.float32)), np.zeros(n_inst, np.int64))
        members = np.concatenate([np.asarray(m, dtype=np.int64) for m, _, _ in groups])
        member_counts = np.concatenate([np.asarray(c, dtype=np.int64) for _, c, _ in groups])
        counts = np.bincount(members, member_counts, minlength=n_inst).astype(np.int64)
        cols = [np.concatenate([g[2][j] for g in groups]) if len(groups) > 1 else g0
                for j, g0 in enumerate(groups[0][2])]
        if np.any(np.diff(members) < 0):  # the groups interleave instances: put the points in instance order
            order = np.argsort(np.repeat(members, member_counts), kind="stable")
            cols = [c[order] for c in cols]
        return cls(cols, counts)

    @staticmethod
    def _dest(sets):
        """Per set, where its points go when each instance takes its points
        of every set in turn; and the combined counts."""
        counts = sum(s.counts for s in sets)
        starts = np.concatenate([[0], np.cumsum(counts)])
        before, dests = np.zeros_like(counts), []
        for s in sets:
            inst = s.inst
            dests.append(starts[inst] + before[inst] + (np.arange(s.n) - s.starts[inst]))
            before = before + s.counts
        return dests, counts

    @classmethod
    def interleave(cls, sets) -> "_PointSets":
        """Per instance, its points of each set in turn (the per-instance
        concatenation of the sets)."""
        dests, counts = cls._dest(sets)
        cols = [np.empty((int(counts.sum()),) + c.shape[1:], c.dtype) for c in sets[0].cols]
        for s, dest in zip(sets, dests):
            for o, c in zip(cols, s.cols):
                o[dest] = c
        return cls(cols, counts)

    @classmethod
    def interleave_values(cls, values, sets) -> np.ndarray:
        """interleave for one per-point array per set."""
        dests, counts = cls._dest(sets)
        out = np.empty(int(counts.sum()), np.asarray(values[0]).dtype)
        for v, dest in zip(values, dests):
            out[dest] = v
        return out


def _limit_rows(row_sizes, caps, rng):
    """Per row r of a ragged list (row_sizes[r] items, rows back to back), at
    most caps[r] items drawn at random (all when they fit), as ascending flat
    indices: _limit for many rows at once."""
    row_sizes = np.asarray(row_sizes, dtype=np.int64)
    total = int(row_sizes.sum())
    if total == 0:
        return np.zeros(0, np.int64)
    row = np.repeat(np.arange(row_sizes.shape[0]), row_sizes)
    order = np.lexsort((rng.random(total), row))
    starts = np.concatenate([[0], np.cumsum(row_sizes)[:-1]])
    rank = np.arange(total) - starts[row[order]]
    return np.sort(order[rank < np.asarray(caps, dtype=np.int64)[row[order]]])


def _audit_sources_group(t, mesh, mats, kernels, caps, edge_list, vertex_list, rng):
    """Boundary-edge points, inset corners, centroids and render vertices of
    the g instances of one mesh at once (t f32[g, T, 3, 3], mats their
    transforms, kernels and caps per instance); one random stream for the
    group. Returns, per instance, the four point sets as 5-tuples."""
    g = t.shape[0]
    out = [[] for _ in range(g)]
    for counts, cols in _audit_sources_group_flat(t, mesh, mats, kernels, caps, edge_list, vertex_list, rng):
        bounds = np.concatenate([[0], np.cumsum(counts)])
        for j in range(g):
            out[j].append(tuple(c[bounds[j]:bounds[j + 1]] for c in cols))
    return out


def _audit_sources_group_flat(t, mesh, mats, kernels, caps, edge_list, vertex_list, rng):
    """_audit_sources_group's four point kinds, each as (points per
    instance, (pos, nrm, tri, b1, b2) back to back in instance order)."""
    g, n_tri = t.shape[0], t.shape[1]
    corners = np.array([[0, 1], [1, 2], [2, 0]])
    out = []

    def emit(pos, nrm, tri, b1, b2, row):
        out.append((np.bincount(row, minlength=g), (pos, nrm, tri, b1, b2)))

    # boundary-edge segment midpoints, spacing R / 2 per instance
    face, local = edge_list
    if face.size:
        a, b = corners[local, 0], corners[local, 1]
        p0, p1 = t[:, face, a], t[:, face, b]  # [g, E, 3]
        spacing = np.maximum(np.asarray(kernels, dtype=np.float64) * 0.5, 1e-8)
        seg = np.maximum(np.ceil(np.linalg.norm(p1 - p0, axis=2) / spacing[:, None]).astype(np.int64), 1)
        flat_seg = seg.reshape(-1)
        edge_of = np.repeat(np.arange(flat_seg.size), flat_seg)  # (instance, edge) per segment
        first = np.concatenate([[0], np.cumsum(flat_seg)[:-1]])
        u = ((np.arange(edge_of.size) - first[edge_of]).astype(np.float32) + np.float32(0.5)) / \
            flat_seg[edge_of].astype(np.float32)
        keep = _limit_rows(seg.sum(axis=1), caps, rng)
        edge_of, u = edge_of[keep], u[keep]
        row, e = edge_of // face.size, edge_of % face.size
        pos = (p0[row, e] * (1.0 - u[:, None]) + p1[row, e] * u[:, None]).astype(np.float32)
        bary = np.zeros((keep.size, 3), np.float32)
        bary[np.arange(keep.size), a[e]] = 1.0 - u
        bary[np.arange(keep.size), b[e]] = u
        emit(pos, _face_normals(t[row, face[e]]), face[e].astype(np.uint32), bary[:, 1], bary[:, 2], row)
    else:
        emit(*(np.zeros((0, 3), np.float32),) * 2, np.zeros(0, np.uint32), *(np.zeros(0, np.float32),) * 2,
             np.zeros(0, np.int64))
    # inset corners (R / 20 inside the face)
    keep = _limit_rows(np.full(g, 3 * n_tri), caps, rng)
    row, c = keep // (3 * n_tri), keep % (3 * n_tri)
    tri, corner = c // 3, c % 3
    ts = t[row, tri]
    edges = np.stack([np.linalg.norm(ts[:, 1] - ts[:, 0], axis=1), np.linalg.norm(ts[:, 2] - ts[:, 1], axis=1),
                      np.linalg.norm(ts[:, 0] - ts[:, 2], axis=1)], axis=1)
    inset_d = (np.asarray(kernels, dtype=np.float64) * 0.05)[row]
    inset = np.clip(inset_d / np.maximum(edges.max(axis=1), 1e-8), 1e-4, 0.1).astype(np.float32)
    bary = np.repeat(inset[:, None], 3, axis=1)
    bary[np.arange(keep.size), corner] = 1.0 - 2.0 * inset
    emit(np.einsum("ni,nij->nj", bary, ts).astype(np.float32), _face_normals(ts), tri.astype(np.uint32),
         bary[:, 1], bary[:, 2], row)
    # centroids
    keep = _limit_rows(np.full(g, n_tri), caps, rng)
    row, tri = keep // n_tri, keep % n_tri
    ts = t[row, tri]
    third = np.full(keep.size, 1.0 / 3.0, np.float32)
    emit(ts.mean(axis=1, dtype=np.float32), _face_normals(ts), tri.astype(np.uint32), third, third, row)
    # render vertices with their transformed normals
    verts, first_slot = vertex_list
    keep = _limit_rows(np.full(g, verts.size), caps, rng)
    row, v = keep // verts.size, keep % verts.size
    m = np.asarray(mats, dtype=np.float64)
    vp = mesh.vertices[verts[v], :3].astype(np.float64)
    vn = mesh.vertices[verts[v], 3:6].astype(np.float64)
    pos = (np.einsum("nk,njk->nj", vp, m[row, :3, :3]) + m[row, :3, 3]).astype(np.float32)
    inv = np.linalg.inv(m[:, :3, :3])
    nrm = np.einsum("nk,nkj->nj", vn, inv[row]).astype(np.float32)
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-20)
    slot = first_slot[v]
    emit(pos, nrm, (slot // 3).astype(np.uint32), (slot % 3 == 1).astype(np.float32),
         (slot % 3 == 2).astype(np.float32), row)
    return out


def _face_normals(t):
    cr = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]).astype(np.float64)
    return (cr / np.maximum(np.linalg.norm(cr, axis=1, keepdims=True), 1e-30)).astype(np.float32)


def _group_centroids(t):
    """Every triangle's centroid and face normal for the g instances of one
    mesh at once (t f32[g, T, 3, 3]): per element the operations of
    _centroids(t[j], T, None), so the values are the same."""
    cen = t.mean(axis=2, dtype=np.float32)
    cr = np.cross(t[:, :, 1] - t[:, :, 0], t[:, :, 2] - t[:, :, 0]).astype(np.float64)
    nrm = (cr / np.maximum(np.linalg.norm(cr, axis=2, keepdims=True), 1e-30)).astype(np.float32)
    return cen, nrm


def _limit(n, k, rng):
    return np.arange(n) if n <= k else np.sort(rng.choice(n, size=k, replace=False))


def _centroids(t, k, rng):
    """Triangle centroids (_triangle_centroid_candidates, :593-611), at most k."""
    idx = _limit(t.shape[0], k, rng)
    third = np.full(idx.shape[0], 1.0 / 3.0, np.float32)
    return (t[idx].mean(axis=1, dtype=np.float32), _face_normals(t)[idx], idx.astype(np.uint32), third, third)


def _inset_corners(t, inset_distance, k, rng):
    """Corners pulled inside their face (_triangle_inset_corner_candidates,
    :614-655), at most k (the subset drawn first, then only it computed)."""
    idx = _limit(3 * t.shape[0], k, rng)
    tri, corner = idx // 3, idx % 3
    ts = t[tri]
    edges = np.stack([np.linalg.norm(ts[:, 1] - ts[:, 0], axis=1), np.linalg.norm(ts[:, 2] - ts[:, 1], axis=1),
                      np.linalg.norm(ts[:, 0] - ts[:, 2], axis=1)], axis=1)
    inset = np.clip(float(inset_distance) / np.maximum(edges.max(axis=1), 1e-8), 1e-4, 0.1).astype(np.float32)
    bary = np.repeat(inset[:, None], 3, axis=1)
    bary[np.arange(idx.shape[0]), corner] = 1.0 - 2.0 * inset
    pos = np.einsum("ni,nij->nj", bary, ts).astype(np.float32)
    return pos, _face_normals(ts), tri.astype(np.uint32), bary[:, 1], bary[:, 2]


def _boundary_edge_list(mesh_indices):
    """(face, local edge) of every edge used by one triangle only, keyed by
    vertex index (_boundary_edge_topology, surface_probes.py:658-688); a
    property of the mesh, shared by its instances."""
    corners = np.array([[0, 1], [1, 2], [2, 0]])
    ev = np.sort(mesh_indices.astype(np.int64)[:, corners].reshape(-1, 2), axis=1)
    keys = ev[:, 0] * (int(ev.max(initial=0)) + 1) + ev[:, 1]
    _, inverse, counts = np.unique(keys, return_inverse=True, return_counts=True)
    edges = np.flatnonzero(counts[inverse] == 1)
    return edges // 3, edges % 3


def _boundary_edges(t, mesh_indices, spacing, edge_list=None):
    """Points along the edges used by one triangle only
    (_boundary_edge_candidates, surface_probes.py:690-779): ceil(length /
    spacing) segment midpoints per edge, with the face normal. edge_list:
    the mesh's _boundary_edge_list, when already known."""
    corners = np.array([[0, 1], [1, 2], [2, 0]])
    face, local = _boundary_edge_list(mesh_indices) if edge_list is None else edge_list
    empty = (np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), np.zeros(0, np.uint32),
             np.zeros(0, np.float32), np.zeros(0, np.float32))
    if face.size == 0:
        return empty
    a, b = corners[local, 0], corners[local, 1]
    p0, p1 = t[face, a], t[face, b]
    seg = np.maximum(np.ceil(np.linalg.norm(p1 - p0, axis=1) / max(float(spacing), 1e-8)).astype(np.int64), 1)
    edge_of = np.repeat(np.arange(face.size), seg)
    first = np.concatenate([[0], np.cumsum(seg)[:-1]])
    step = (np.arange(edge_of.size) - first[edge_of]).astype(np.float32)
    u = (step + np.float32(0.5)) / seg[edge_of].astype(np.float32)
    pos = (p0[edge_of] * (1.0 - u[:, None]) + p1[edge_of] * u[:, None]).astype(np.float32)
    bary = np.zeros((edge_of.size, 3), np.float32)
    rows = np.arange(edge_of.size)
    bary[rows, a[edge_of]] = 1.0 - u
    bary[rows, b[edge_of]] = u
    return pos, _face_normals(t[face])[edge_of], face[edge_of].astype(np.uint32), bary[:, 1], bary[:, 2]


def _vertex_list(mesh):
    """The mesh's used vertices and, for each, the first index slot naming
    it (a property of the mesh, shared by its instances)."""
    flat_idx = mesh.indices.astype(np.int64).reshape(-1)
    return np.unique(flat_idx, return_index=True)


def _render_vertices(mesh, transform, k, rng, vertex_list=None):
    """The instance's render vertices with their transformed normals, each on
    its first incident triangle (_instance_vertex_anchors,
    surface_probes.py:375-442), at most k."""
    verts, first = _vertex_list(mesh) if vertex_list is None else vertex_list
    idx = _limit(verts.shape[0], k, rng)
    verts, first = verts[idx], first[idx]
    m = np.asarray(transform, dtype=np.float64)
    pos = (mesh.vertices[verts, :3].astype(np.float64) @ m[:3, :3].T + m[:3, 3]).astype(np.float32)
    nrm = (mesh.vertices[verts, 3:6].astype(np.float64) @ np.linalg.inv(m[:3, :3])).astype(np.float32)
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-20)
    tri, corner = first // 3, first % 3
    return pos, nrm, tri.astype(np.uint32), (corner == 1).astype(np.float32), (corner == 2).astype(np.float32)


def _instance_areas(scene_node, chunk_triangles: int = 1 << 20):
    """Per instance: world-space surface area (float64: transformed
    vertices, |cross| / 2 summed over its triangles) and triangle count. The
    instances of one mesh are transformed together, in chunks of about
    chunk_triangles triangles; each instance's arithmetic is the one its own
    transform alone would do."""
    n = len(scene_node.instances)
    areas = np.zeros(n)
    tri_counts = np.zeros(n, np.int64)
    groups: dict = {}
    for i, (mesh_id, _, _) in enumerate(scene_node.instances):
        groups.setdefault(mesh_id, []).append(i)
    for mesh_id, members in groups.items():
        mesh = scene_node.meshes[mesh_id]
        v = mesh.vertices[:, :3].astype(np.float64)
        idx = mesh.indices.astype(np.int64).reshape(-1, 3)
        step = max(1, chunk_triangles // max(idx.shape[0], 1))
        for c in range(0, len(members), step):
            part = members[c:c + step]
            m = np.stack([np.asarray(scene_node.transforms[scene_node.instances[i][2]], dtype=np.float64)
                          for i in part])
            t = (v @ m[:, :3, :3].transpose(0, 2, 1) + m[:, None, :3, 3])[:, idx]  # [g, T, 3, 3]
            cr = np.cross(t[:, :, 1] - t[:, :, 0], t[:, :, 2] - t[:, :, 0])
            areas[part] = 0.5 * np.linalg.norm(cr, axis=2).sum(axis=1)
            tri_counts[part] = idx.shape[0]
    return areas, tri_counts



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
    # per-instance build statistics under the reference's
    # SurfaceProbeInstanceInfo names (surface_probes.py:131-165)
    base_surface_site_count: int = 0
    repair_surface_site_count: int = 0
    protected_surface_site_count: int = 0
    candidate_count: int = 0
    audit_point_count: int = 0
    vertex_anchor_site_count: int = 0
    vertex_anchor_probe_count: int = 0


@dataclass(frozen=True)
class SurfaceProbeSiteLayout:
    probes: np.ndarray
    nodes: np.ndarray
    triangle_vertex_probes: np.ndarray
    instance_gpu_data: np.ndarray
    instance_infos: tuple
    total_probe_count: int
    max_density_multiplier: float
    # build statistics under the reference's SurfaceProbeLayout names
    # (surface_probes.py:1490-1533); build_wse fills them
    target_surface_site_count: int = 0
    total_base_surface_site_count: int = 0
    total_repair_surface_site_count: int = 0
    total_protected_surface_site_count: int = 0
    repair_surface_site_budget: int = 0
    total_surface_site_count: int = 0
    total_candidate_count: int = 0
    total_audit_point_count: int = 0
    zero_gather_before: int = 0
    zero_gather_after_repair: int = 0
    zero_gather_after: int = 0
    deficit_point_count_before: int = 0
    deficit_point_count_after_repair: int = 0
    deficit_point_count_after: int = 0
    ess_p50_before: float = 0.0
    ess_p50_after: float = 0.0
    support_f_p10: float = 0.0
    support_f_p50: float = 0.0
    density_m_p95: float = 0.0
    adaptive_wse: bool = False
    density_driven: bool = False
    density_scale: float = 1.0
    total_surface_area: float = 0.0
    total_adaptive_mass: float = 0.0
    total_vertex_anchor_site_count: int = 0
    total_vertex_anchor_probe_count: int = 0
    oversample_factor: int = 0
    seed: int = 0

    @classmethod
    def from_sites(cls, scene_node, probes, *, leaf_capacity: int = 8, max_depth: int = 16,
                   kernel_radius_scale: float = 2.5, normal_angle_degrees: float = 45.0,
                   max_density_multiplier: float = 8.0, poisson_radii=None,
                   kernel_radii=None, vertex_anchors=None, sampler=None,
                   instance_stats=None, instance_areas=None) -> "SurfaceProbeSiteLayout":
        """instance_stats (optional): further SurfaceProbeSiteInstance fields
        as {name: one value per instance}, e.g. a site builder's counts.
        instance_areas (optional): each instance's surface area when the
        caller has it already (else from the scene's transformed triangles).

        vertex_anchors (optional, per instance None or (records, map,
        anchor site count)): anchor probe records (fronts, then backs for a
        double-sided instance) kept after the instance's octree-ordered probes
        and outside its octree, and map u32[T, 3] naming each triangle's three
        vertex anchors (0xFFFFFFFF: none); the packed triangle map then points
        each triangle side at its anchors (surface_probes.py:2712-2758).
        With a SurfaceProbeSampler the instances' octrees are built on its
        GPU in one call (nan_build_point_octrees), else by
        build_point_octree on the host; both give the same nodes and order."""
        probes = np.asarray(probes, dtype=SURFACE_PROBE_DTYPE)
        instance_of = (probes["meta"][:, 3] >> SURFACE_PROBE_INSTANCE_SHIFT).astype(np.int64)
        n_inst = len(scene_node.instances)
        if probes.shape[0] and int(instance_of.max()) >= n_inst:
            raise ValueError("a probe names an instance the scene does not have")
        if instance_areas is None:
            areas, tri_counts = _instance_areas(scene_node)
        else:
            areas = np.asarray(instance_areas, dtype=np.float64).reshape(-1)
            mesh_tris = [m.indices.reshape(-1, 3).shape[0] for m in scene_node.meshes]
            tri_counts = np.array([mesh_tris[mesh_id] for mesh_id, _, _ in scene_node.instances], np.int64)
        fronts = np.bincount(instance_of[(probes["meta"][:, 3] & 1) == 0], minlength=n_inst)
        total_sites = max(int(fronts.sum()), 1)
        global_kernel = max(math.sqrt(max(float(areas.sum()), 1e-20) / total_sites) * kernel_radius_scale, 1e-5)
        normal_cos = math.cos(math.radians(normal_angle_degrees))
        if kernel_radii is not None:
            kernel = np.asarray(kernel_radii, dtype=np.float64).reshape(-1)[:n_inst]
        else:
            with np.errstate(divide="ignore", invalid="ignore"):
                per_site = np.where(fronts > 0, np.sqrt(areas / np.maximum(fronts, 1)) * kernel_radius_scale, 0.0)
            kernel = np.maximum(np.maximum(global_kernel, per_site), 1e-5)
            if poisson_radii is not None:
                kernel = np.maximum(kernel, np.asarray(poisson_radii, dtype=np.float64).reshape(-1)[:n_inst] *
                                    kernel_radius_scale)

        # the records grouped by instance, each group in its octree's order
        by_instance = np.argsort(instance_of, kind="stable")
        counts = np.bincount(instance_of, minlength=n_inst).astype(np.int64)
        starts = np.concatenate([[0], np.cumsum(counts)])
        rec_all = probes[by_instance]
        inst_sorted = instance_of[by_instance]
        rec_all["position_radius"][:, 3] = kernel[inst_sorted]
        roots = np.zeros((n_inst, 4), np.float64)
        if sampler is not None and probes.shape[0]:
            tree_nodes, tree_node_offsets, order, roots[:] = sampler.build_point_octrees_flat(
                rec_all["position_radius"][:, :3], starts, leaf_capacity=leaf_capacity, max_depth=max_depth)
            node_counts = np.diff(tree_node_offsets.astype(np.int64))
        else:
            parts, order_parts = [], []
            node_counts = np.zeros(n_inst, np.int64)
            for i in np.flatnonzero(counts):
                nodes, order_i, center, extent = build_point_octree(
                    rec_all["position_radius"][starts[i]:starts[i + 1], :3], leaf_capacity=leaf_capacity,
                    max_depth=max_depth)
                parts.append(nodes)
                order_parts.append(order_i)
                node_counts[i] = nodes.shape[0]
                roots[i] = (*center, extent)
            tree_nodes = np.concatenate(parts) if parts else np.zeros((0, 4), np.uint32)
            order = np.concatenate(order_parts) if order_parts else np.zeros(0, np.int64)
        node_counts[counts == 0] = 0
        roots[counts == 0] = 0.0
        rec_all = rec_all[starts[inst_sorted] + order]
        # anchor records follow their instance's octree records
        anchor_counts = np.zeros(n_inst, np.int64)
        anchored = [] if vertex_anchors is None else [i for i in range(n_inst) if vertex_anchors[i] is not None]
        for i in anchored:
            anchor_counts[i] = np.asarray(vertex_anchors[i][0]).shape[0]
        rec_counts = counts + anchor_counts
        probe_offsets = np.concatenate([[0], np.cumsum(rec_counts)])
        node_offsets = np.concatenate([[0], np.cumsum(node_counts)])
        map_offsets = np.concatenate([[0], np.cumsum(tri_counts * 2)])
        if anchored:
            out_probes = np.zeros(int(probe_offsets[-1]), dtype=SURFACE_PROBE_DTYPE)
            out_probes[probe_offsets[inst_sorted] + (np.arange(inst_sorted.shape[0]) - starts[inst_sorted])] = rec_all
        else:
            out_probes = rec_all
        nodes_all = np.ascontiguousarray(tree_nodes, np.uint32).copy()
        node_inst = np.repeat(np.arange(n_inst), node_counts)
        branch = nodes_all[:, 1] != 0
        nodes_all[branch, 0] += node_offsets[node_inst[branch]].astype(np.uint32)
        nodes_all[~branch, 2] += probe_offsets[node_inst[~branch]].astype(np.uint32)
        maps_all = np.full((int(map_offsets[-1]), 4), 0xFFFFFFFF, np.uint32)
        maps_all[:, 3] = 0
        for i in anchored:
            anchor_rec, tri_map, anchor_sites = vertex_anchors[i]
            anchor_rec = np.asarray(anchor_rec, dtype=SURFACE_PROBE_DTYPE).copy()
            anchor_rec["position_radius"][:, 3] = kernel[i]
            first = int(probe_offsets[i] + counts[i])
            out_probes[first:first + anchor_rec.shape[0]] = anchor_rec
            tri_map = np.asarray(tri_map, dtype=np.uint32).reshape(-1, 3)
            valid = np.flatnonzero(np.all(tri_map != 0xFFFFFFFF, axis=1))
            front = tri_map[valid] + np.uint32(first)
            back = front + np.uint32(anchor_sites) if anchor_rec.shape[0] > anchor_sites else front
            maps = maps_all[map_offsets[i]:map_offsets[i + 1]]
            maps[2 * valid, :3] = front
            maps[2 * valid + 1, :3] = back
            maps[2 * valid, 3] |= 1
            maps[2 * valid + 1, 3] |= 1

        plane_sigma = np.maximum(kernel * 0.25, 1e-6)
        gpu = np.zeros(n_inst, dtype=SURFACE_PROBE_INSTANCE_DTYPE)
        gpu["root_center_extent"] = roots
        gpu["offsets"] = np.stack([node_offsets[:-1], node_counts, probe_offsets[:-1], rec_counts],
                                  axis=1).astype(np.uint32)
        gpu["params"][:, 0] = kernel
        gpu["params"][:, 1] = normal_cos
        gpu["params"][:, 2] = plane_sigma
        gpu["params"][:, 3] = map_offsets[:-1].astype(np.uint32).view(np.float32)
        roots_l, kernel_l, sigma_l, areas_l = roots.tolist(), kernel.tolist(), plane_sigma.tolist(), areas.tolist()
        stats = instance_stats or {}
        stat_l = {k: np.asarray(v).tolist() for k, v in stats.items()}
        infos = tuple(
            SurfaceProbeSiteInstance(tuple(roots_l[i][:3]), roots_l[i][3], no, nc, po, pc, kernel_l[i], normal_cos,
                                     sigma_l[i], areas_l[i], fr, co, **{k: v[i] for k, v in stat_l.items()})
            for i, (no, nc, po, pc, fr, co) in enumerate(zip(node_offsets[:-1].tolist(), node_counts.tolist(),
                                                             probe_offsets[:-1].tolist(), rec_counts.tolist(),
                                                             fronts.tolist(), counts.tolist())))
        all_nodes = nodes_all if nodes_all.shape[0] else np.zeros((1, 4), np.uint32)
        all_maps = maps_all if maps_all.shape[0] else np.zeros((2, 4), np.uint32)
        return cls(out_probes, np.ascontiguousarray(all_nodes, np.uint32), np.ascontiguousarray(all_maps, np.uint32),
                   gpu, infos, int(probe_offsets[-1]), float(max_density_multiplier))

    @classmethod
    def build_wse(cls, scene_node, target_probe_count: int, *, device=None, oversample_factor: int = 5,
                  seed: int = 1, minimum_per_instance: int = 4, repair_budget_ratio: float = 0.30,
                  repair_min_gather: int = 4, kernel_radius_scale: float = 2.5, normal_angle_degrees: float = 45.0,
                  adaptive_wse: bool = True, max_density_multiplier: float = 8.0,
                  build_vertex_anchors: bool = False, adaptive_mass_site_density: float | None = None,
                  density_reference_kernel_radius: float | None = None, density_scale: float = 1.0,
                  sampler=None, profile: dict | None = None, **kwargs) -> "SurfaceProbeSiteLayout":
        """Sites by weighted sample elimination of oversampled candidates, then
        deficit repair: audit points (filtered from boundary-edge points, inset
        corners, centroids, the candidates, a second surface sample and the
        render vertices per instance) that gather
        fewer than repair_min_gather sites get repair sites from the filtered
        repair candidates, up to repair_budget_ratio x the target; audit
        points still short then get their residual deficit as colocated
        protected sites, without a budget (the protected closure; its sites
        carry SURFACE_PROBE_FLAG_PROTECTED). repair_min_gather = 0 turns
        repair and closure off.

        adaptive_wse (the reference's default, surface_probes.py:1706-2000)
        first measures each triangle's support f at its centroid against a
        surface sample plus every centroid (radius: the global kernel
        radius) and gives it the density m = min(M, 1 / max(f, 1/M)); the
        instance budget then follows area x m, candidates are drawn with
        probability proportional to area x m, and the elimination is the
        adaptive one with each candidate's relative density
        m / (adaptive mass / area).

        build_vertex_anchors (off by default, as in the reference) adds one
        anchor probe per render vertex of each instance, flagged
        SURFACE_PROBE_FLAG_VERTEX_ANCHOR and kept outside the octree, and
        the triangle map the resolve's vertex fallback reads.

        Density mode (target_probe_count None, with adaptive_mass_site_density
        and density_reference_kernel_radius; surface_probes.py:1588-1626,
        1838-1866): the kernel radius is the reference radius /
        sqrt(density_scale) and each instance gets floor(adaptive mass x
        density x scale + 0.5) + repair_min_gather sites, so the total is an
        output of the world-space density."""
        import time

        from .surface_probe_sampler import SurfaceProbeSampler

        t0 = time.perf_counter()
        # world triangles and areas, the instances of one mesh transformed together
        n_inst = len(scene_node.instances)
        tris, areas = [None] * n_inst, [None] * n_inst
        double_sided = [bool(scene_node.materials[mat_id].double_sided) for _, mat_id, _ in scene_node.instances]
        by_mesh: dict = {}
        group_geometry: dict = {}
        group_normals: dict = {}
        for i, (mesh_id, _, _) in enumerate(scene_node.instances):
            by_mesh.setdefault(mesh_id, []).append(i)
        for mesh_id, members in by_mesh.items():
            mesh = scene_node.meshes[mesh_id]
            mats = np.stack([np.asarray(scene_node.transforms[scene_node.instances[i][2]], dtype=np.float64)
                             for i in members])
            p = np.einsum("vk,gjk->gvj", mesh.vertices[:, :3].astype(np.float64), mats[:, :3, :3]) + \
                mats[:, None, :3, 3]
            t = p[:, mesh.indices.astype(np.int64)].astype(np.float32)  # [g, T, 3, 3]
            e = np.cross(t[:, :, 1] - t[:, :, 0], t[:, :, 2] - t[:, :, 0]).astype(np.float64)
            norm_e = np.linalg.norm(e, axis=2)
            a = 0.5 * norm_e
            # face normals as _face_normals forms them, kept for every sampled point
            group_normals[mesh_id] = (e / np.maximum(norm_e[..., None], 1e-30)).astype(np.float32)
            group_geometry[mesh_id] = (t, a)
            for j, i in enumerate(members):
                tris[i], areas[i] = t[j], a[j]

        # each instance's triangles at tri_starts[i] in per-triangle arrays
        tri_starts = np.concatenate([[0], np.cumsum([t.shape[0] for t in tris])]).astype(np.int64)

        def group_rows(values, members):
            """[g, T] rows of a per-triangle array for the instances of one mesh."""
            return values[tri_starts[np.asarray(members)][:, None] + np.arange(tris[members[0]].shape[0])]

        def sample_by_mesh(per_instance, salt, densities=None):
            """Area (x density) weighted surface points of every instance, the
            instances of one mesh drawn together from one stream; densities
            per triangle (all instances' triangles back to back) or None."""
            per_instance = np.asarray(per_instance, dtype=np.int64)
            groups = []
            for mesh_id, members in by_mesh.items():
                t, a = group_geometry[mesh_id]
                dens = None if densities is None else group_rows(densities, members)
                rng = np.random.default_rng([int(seed), int(mesh_id), int(salt)])
                groups.append((members, per_instance[members],
                               _surface_points_group_flat(t, a, per_instance[members], rng, dens,
                                                          normals=group_normals[mesh_id])))
            return _PointSets.from_groups(groups, n_inst)

        totals = np.zeros(n_inst)
        for mesh_id, members in by_mesh.items():
            totals[members] = group_geometry[mesh_id][1].sum(axis=1)
        density_driven = target_probe_count is None
        if density_driven:
            if adaptive_mass_site_density is None or density_reference_kernel_radius is None:
                raise ValueError("Surface probes require an explicit count or density mode")
            if not (math.isfinite(density_scale) and density_scale > 0.0 and
                    math.isfinite(adaptive_mass_site_density) and adaptive_mass_site_density > 0.0 and
                    math.isfinite(density_reference_kernel_radius) and density_reference_kernel_radius > 0.0):
                raise ValueError("density mode needs finite, positive density, kernel radius and scale")
            global_kernel = max(float(density_reference_kernel_radius) / math.sqrt(density_scale), 1e-5)
            spacing = global_kernel / kernel_radius_scale
            minimum = max(1, int(repair_min_gather))
            counts = allocate_density_counts(totals, 1.0 / max(spacing * spacing, 1e-20), minimum_per_entry=minimum)
            target = int(counts.sum())
        else:
            target = int(target_probe_count)
            minimum = min(minimum_per_instance, max(1, target // max(len(totals), 1)))
            counts = allocate_counts(totals, target, minimum_per_entry=minimum)
            global_kernel = max(math.sqrt(max(float(totals.sum()), 1e-20) / max(target, 1)) * kernel_radius_scale,
                                1e-5)
        if sampler is None:
            from .scene import Device

            sampler = SurfaceProbeSampler(device if device is not None else Device(0))
        ncos = math.cos(math.radians(normal_angle_degrees))
        tri_density = None  # per triangle, all instances back to back
        t_pre = time.perf_counter()
        if adaptive_wse:
            n_refs = np.clip(np.asarray(counts, dtype=np.int64) * min(max(1, int(oversample_factor)), 2), 1, 131072)
            rnds = sample_by_mesh(n_refs, 17)
            cen_groups, half_area = [], []
            for mesh_id, members in by_mesh.items():
                t_g, a_g = group_geometry[mesh_id]
                cm, cn = t_g.mean(axis=2, dtype=np.float32), group_normals[mesh_id]  # as _group_centroids
                g, n_tri = a_g.shape
                third = np.full(g * n_tri, 1.0 / 3.0, np.float32)
                cen_groups.append((members, np.full(g, n_tri), (cm.reshape(-1, 3), cn.reshape(-1, 3),
                                                                np.tile(np.arange(n_tri, dtype=np.uint32), g), third,
                                                                third)))
                half_area.append((members, np.full(g, n_tri), ((0.5 * a_g).astype(np.float32).reshape(-1),)))
            cens = _PointSets.from_groups(cen_groups, n_inst)
            rnd_w = np.repeat((0.5 * totals / np.maximum(rnds.counts, 1)).astype(np.float32), rnds.counts)
            ref_w = _PointSets.interleave_values([rnd_w, _PointSets.from_groups(half_area, n_inst).cols[0]],
                                                 [rnds, cens])
            refs = _PointSets.interleave([rnds, cens])
            _, tri_density = sampler.estimate_support(refs.cols[0], refs.cols[1], refs.inst, ref_w, cens.cols[0],
                                                      cens.cols[1], cens.inst,
                                                      np.full(n_inst, global_kernel, np.float32),
                                                      normal_cosine_threshold=ncos,
                                                      max_density_multiplier=max_density_multiplier)
            masses = np.zeros(n_inst)
            for mesh_id, members in by_mesh.items():
                a_g = group_geometry[mesh_id][1]
                masses[members] = (a_g * group_rows(tri_density, members).astype(np.float64)).sum(axis=1)
            if density_driven:
                counts = allocate_density_counts(masses, float(adaptive_mass_site_density) * float(density_scale),
                                                 minimum_per_entry=minimum)
                target = int(counts.sum())
            else:
                counts = allocate_counts(masses, target, minimum_per_entry=minimum)
        elif density_driven:
            counts = allocate_density_counts(totals, float(adaptive_mass_site_density) * float(density_scale),
                                             minimum_per_entry=minimum)
            target = int(counts.sum())
        t_pre_end = time.perf_counter()
        counts = np.asarray(counts, dtype=np.int64)
        cands = sample_by_mesh(counts * max(1, int(oversample_factor)), 0, tri_density if adaptive_wse else None)
        offsets = cands.starts
        cand_density = None
        if adaptive_wse:
            # a candidate's density over its instance's mean density (mass /
            # area, at least 1e-6: below it the float32 quotient by 1e-6)
            ratio = masses / np.maximum(totals, 1e-30)
            inst = cands.inst
            d = tri_density[tri_starts[inst] + cands.cols[2]]
            cand_density = (d / np.maximum(ratio, 1e-6)[inst]).astype(np.float32)
            low = (ratio < 1e-6)[inst]
            if low.any():
                cand_density[low] = d[low] / np.float32(1e-6)
        t1 = time.perf_counter()
        keep, radii = sampler.eliminate(cands.cols[0], cands.cols[1], offsets, counts, totals,
                                        relative_densities=cand_density)
        keep = keep.cpu().numpy().astype(bool)
        t2 = time.perf_counter()
        base_sel = np.flatnonzero(keep)
        sites = cands.take(base_sel)
        flags = np.zeros(sites.n, np.uint32)
        repaired = protected = 0
        budget = int(math.floor(target * float(repair_budget_ratio)))
        # kernel radius per instance, fixed before the repair as the reference does
        kernels = np.maximum.reduce([np.full(n_inst, global_kernel),
                                     np.sqrt(totals / np.maximum(counts, 1)) * kernel_radius_scale,
                                     np.asarray(radii, dtype=np.float64) * kernel_radius_scale,
                                     np.full(n_inst, 1e-5)]).astype(np.float32)
        stats: dict = {}
        per_repair = per_protected = per_audit = np.zeros(n_inst, np.int64)
        if repair_min_gather > 0:
            # audit source per instance (surface_probes.py:2026-2180): boundary
            # edge points, inset corners, centroids, every base candidate, a
            # second surface sample and the render vertices; the filter keeps
            # one audit point per cell of R/2 and normal cone, and as repair
            # candidates those that no selected base site or earlier
            # candidate duplicates bit for bit
            seconds = sample_by_mesh(counts, 7919)
            kinds = [[] for _ in range(4)]  # boundary, inset, centroid, vertices
            for mesh_id, members in by_mesh.items():
                mesh = scene_node.meshes[mesh_id]
                mats = np.stack([np.asarray(scene_node.transforms[scene_node.instances[i][2]], dtype=np.float64)
                                 for i in members])
                parts = _audit_sources_group_flat(group_geometry[mesh_id][0], mesh, mats, kernels[members],
                                                  np.maximum(16, counts[members]), _boundary_edge_list(mesh.indices),
                                                  _vertex_list(mesh),
                                                  np.random.default_rng([int(seed), int(mesh_id), 7919, 1]))
                for kind, (c, cols) in zip(kinds, parts):
                    kind.append((members, c, cols))
            boundary, inset, centroid, vertices = (_PointSets.from_groups(k, n_inst) for k in kinds)
            sources = _PointSets.interleave([boundary, inset, centroid, cands, seconds, vertices])
            filt = sampler.filter_audit_repair_candidates(
                sources.cols[0], sources.cols[1], cands.cols[0], cands.cols[1], base_sel,
                audit_cell_size=(kernels.astype(np.float64) * 0.5), normal_cosine_threshold=ncos,
                candidate_sets=sources.inst, base_sets=cands.inst)
            audits = sources.take(filt.audit_indices)
            repairs = sources.take(filt.repair_indices)
            result = sampler.deficit_repair(sites.cols[0], sites.cols[1], sites.inst, repairs.cols[0],
                                            repairs.cols[1], repairs.inst, audits.cols[0], audits.cols[1],
                                            audits.inst, kernels, min_gather_count=repair_min_gather,
                                            max_repair_count=budget, normal_cosine_threshold=ncos)
            chosen = repairs.take(np.sort(result.selected_candidate_indices))
            per_repair = chosen.counts
            per_audit = audits.counts
            flags = _PointSets.interleave_values([flags, np.zeros(chosen.n, np.uint32)], [sites, chosen])
            sites = _PointSets.interleave([sites, chosen])
            repaired = chosen.n
            # protected closure (surface_probes.py:2462-2587): every audit point
            # still short of the gather target offers its residual deficit as
            # colocated candidates, chosen without a budget
            deficits = np.maximum(int(repair_min_gather) - result.counts_after.astype(np.int64), 0)
            short = np.flatnonzero(deficits)
            closure_after = result.counts_after.copy()
            if short.size:
                audit_inst = audits.inst
                offers = np.repeat(short, deficits[short])
                prot = tuple(c[offers] for c in audits.cols)
                prot_inst = audit_inst[offers]
                closure = sampler.deficit_repair(
                    sites.cols[0], sites.cols[1], sites.inst, prot[0], prot[1], prot_inst,
                    audits.cols[0][short], audits.cols[1][short], audit_inst[short], kernels,
                    min_gather_count=repair_min_gather, max_repair_count=int(offers.shape[0]),
                    normal_cosine_threshold=ncos)
                picked = np.sort(closure.selected_candidate_indices)
                # offers follow the instances, so the picked ones do too
                taken = _PointSets((c[picked] for c in prot), np.bincount(prot_inst[picked], minlength=n_inst))
                per_protected = taken.counts
                flags = _PointSets.interleave_values(
                    [flags, np.full(taken.n, SURFACE_PROBE_FLAG_PROTECTED, np.uint32)], [sites, taken])
                sites = _PointSets.interleave([sites, taken])
                protected = taken.n
                closure_after[short] = closure.counts_after
            stats.update(total_audit_point_count=int(result.counts_before.shape[0]),
                         zero_gather_before=int((result.counts_before == 0).sum()),
                         zero_gather_after_repair=int((result.counts_after == 0).sum()),
                         zero_gather_after=int((closure_after == 0).sum()),
                         deficit_point_count_before=int((result.counts_before < repair_min_gather).sum()),
                         deficit_point_count_after_repair=int((result.counts_after < repair_min_gather).sum()),
                         deficit_point_count_after=int((closure_after < repair_min_gather).sum()),
                         ess_p50_before=float(np.median(result.ess_before)) if result.ess_before.size else 0.0,
                         ess_p50_after=float(np.median(result.ess_after)) if result.ess_after.size else 0.0)
            if profile is not None:
                profile.update(repair_sites=repaired, protected_sites=protected,
                               audits=int(result.counts_before.shape[0]),
                               repair_candidates=int(filt.repair_indices.shape[0]),
                               audits_below_min_before=int((result.counts_before < repair_min_gather).sum()),
                               audits_below_min_after_repair=int((result.counts_after < repair_min_gather).sum()),
                               audits_below_min_after=int((closure_after < repair_min_gather).sum()),
                               zero_gather_after=int((closure_after == 0).sum()),
                               repair_rounds=int(result.rounds))
        t3 = time.perf_counter()
        # support f of every site against the candidate population: area /
        # candidates each, or, for density-drawn candidates, area x
        # (1 / density) normalised to the instance area
        cand_inst = cands.inst
        if adaptive_wse:
            w = 1.0 / np.maximum(tri_density[tri_starts[cand_inst] + cands.cols[2]].astype(np.float64), 1e-12)
            # each instance's sum as numpy forms it for the instance alone
            w_sum = np.array([w[b:e].sum() for b, e in zip(offsets[:-1].tolist(), offsets[1:].tolist())])
            ref_area = (w * (totals / np.maximum(w_sum, 1e-30))[cand_inst]).astype(np.float32)
        else:
            ref_area = np.repeat((totals / np.maximum(cands.counts, 1)).astype(np.float32), cands.counts)
        support, density = sampler.estimate_support(cands.cols[0], cands.cols[1], cand_inst, ref_area,
                                                    sites.cols[0], sites.cols[1], sites.inst, kernels,
                                                    normal_cosine_threshold=ncos,
                                                    max_density_multiplier=max_density_multiplier)
        t4 = time.perf_counter()
        # records per instance: its sites' fronts, then their backs when double-sided
        site_inst = sites.inst
        sides = 1 + np.asarray(double_sided, dtype=np.int64)
        rec_starts = np.concatenate([[0], np.cumsum(sites.counts * sides)])
        local = np.arange(sites.n) - sites.starts[site_inst]
        records = np.zeros(int(rec_starts[-1]), dtype=SURFACE_PROBE_DTYPE)
        inst_bits = site_inst.astype(np.uint32) << np.uint32(SURFACE_PROBE_INSTANCE_SHIFT)
        back = sides[site_inst] == 2
        for side, sel, dest in ((0, slice(None), rec_starts[site_inst] + local),
                                (1, back, (rec_starts[site_inst] + sites.counts[site_inst] + local)[back])):
            pos, nrm, tri, b1, b2 = (c[sel] for c in sites.cols)
            records["position_radius"][dest, :3] = pos
            records["normal_side"][dest, :3] = nrm * np.float32(-1.0) if side else nrm
            records["normal_side"][dest, 3] = support[sel]
            records["meta"][dest, 0] = tri
            records["meta"][dest, 1] = b1.view(np.uint32)
            records["meta"][dest, 2] = b2.view(np.uint32)
            records["meta"][dest, 3] = np.uint32(side) | flags[sel] | inst_bits[sel]
        anchors = None
        if build_vertex_anchors:
            anchors = []
            for i, (mesh_id, _, transform_id) in enumerate(scene_node.instances):
                mesh = scene_node.meshes[mesh_id]
                pos, nrm, tri, b1, b2 = _render_vertices(mesh, scene_node.transforms[transform_id], 1 << 62, None)
                verts = np.unique(mesh.indices.astype(np.int64).reshape(-1))
                lookup = np.full(mesh.vertex_count, 0xFFFFFFFF, np.uint32)
                lookup[verts] = np.arange(verts.shape[0], dtype=np.uint32)
                recs = []
                for side in range(2 if double_sided[i] else 1):
                    r = np.zeros(pos.shape[0], dtype=SURFACE_PROBE_DTYPE)
                    r["position_radius"][:, :3] = pos
                    r["normal_side"][:, :3] = nrm * (-1.0 if side else 1.0)
                    r["normal_side"][:, 3] = 1.0
                    r["meta"][:, 0] = tri
                    r["meta"][:, 1] = b1.view(np.uint32)
                    r["meta"][:, 2] = b2.view(np.uint32)
                    r["meta"][:, 3] = ((1 if side else 0) | SURFACE_PROBE_FLAG_VERTEX_ANCHOR
                                       | (i << SURFACE_PROBE_INSTANCE_SHIFT))
                    recs.append(r)
                anchors.append((np.concatenate(recs), lookup[mesh.indices.astype(np.int64)], pos.shape[0]))
        n_anchor_sites = sum(int(a[2]) for a in anchors) if anchors else 0
        zeros = np.zeros(n_inst, np.int64)
        instance_stats = dict(
            base_surface_site_count=counts, repair_surface_site_count=per_repair,
            protected_surface_site_count=per_protected, candidate_count=cands.counts, audit_point_count=per_audit,
            vertex_anchor_site_count=np.array([a[2] for a in anchors], np.int64) if anchors else zeros,
            vertex_anchor_probe_count=np.array([a[0].shape[0] for a in anchors], np.int64) if anchors else zeros)
        layout = cls.from_sites(scene_node, records, kernel_radii=kernels,
                                normal_angle_degrees=normal_angle_degrees,
                                max_density_multiplier=max_density_multiplier, vertex_anchors=anchors,
                                sampler=sampler, instance_stats=instance_stats, instance_areas=totals, **kwargs)
        layout = dataclasses.replace(
            layout, target_surface_site_count=target, total_base_surface_site_count=int(sum(counts)),
            total_repair_surface_site_count=repaired, total_protected_surface_site_count=protected,
            repair_surface_site_budget=budget if repair_min_gather > 0 else 0,
            total_surface_site_count=sites.n, total_candidate_count=int(offsets[-1]),
            support_f_p10=float(np.percentile(support, 10)) if support.size else 0.0,
            support_f_p50=float(np.median(support)) if support.size else 0.0,
            density_m_p95=float(np.percentile(density, 95)) if density.size else 0.0,
            adaptive_wse=bool(adaptive_wse), density_driven=bool(density_driven),
            density_scale=float(density_scale) if density_driven else 1.0, total_surface_area=float(totals.sum()),
            total_adaptive_mass=float(masses.sum()) if adaptive_wse else float(totals.sum()),
            total_vertex_anchor_site_count=n_anchor_sites,
            total_vertex_anchor_probe_count=int(sum(a[0].shape[0] for a in anchors)) if anchors else 0,
            oversample_factor=int(oversample_factor), seed=int(seed), **stats)
        if profile is not None:
            profile.update(density_prepass_s=t_pre_end - t_pre, adaptive=bool(adaptive_wse),
                           candidates_s=t1 - t0, elimination_s=t2 - t1, repair_s=t3 - t2, support_s=t4 - t3,
                           packing_s=time.perf_counter() - t4, candidates=int(offsets[-1]),
                           rounds=int(sampler.last_rounds), base_sites=int(sum(counts)), repair_sites=repaired,
                           protected_sites=protected,
                           support_p10=float(np.percentile(support, 10)) if support.size else 0.0,
                           support_p50=float(np.median(support)) if support.size else 0.0,
                           density_p95=float(np.percentile(density, 95)) if density.size else 0.0)
        return layout

    @classmethod
    def build(cls, scene_node, site_count: int, *, seed: int = 1, **kwargs) -> "SurfaceProbeSiteLayout":
        """Area-weighted random sites (scenes.surface_sites) packed by from_sites."""
        from .scenes import surface_sites

        probes, _ = surface_sites(scene_node, site_count, seed=seed)
        return cls.from_sites(scene_node, probes, **kwargs)

    def query_probe_indices(self, instance_index: int, position, radius: float | None = None, normal=None):
        return query_probe_indices(self, instance_index, position, radius, normal)


class SurfaceProbeLayout(SurfaceProbeSiteLayout):
    """The reference's SurfaceProbeLayout name and build signature
    (surface_probes.py:1536-1560): build() is build_wse with the reference's
    keywords (sampler_backend and profile_build are accepted and ignored:
    the passes run on the GPU)."""

    @classmethod
    def build(cls, scene_node, *, target_probe_count: int | None = 8192, device=None, sampler_backend=None,
              profile_build: bool = False, **kwargs) -> "SurfaceProbeLayout":
        return cls.build_wse(scene_node, target_probe_count, device=device, **kwargs)
