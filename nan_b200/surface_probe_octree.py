"""Per-instance point octree over surface-probe positions
(_build_point_octree_python, surface_probes.py:1348-1438 of the reference;
the same layout as its C++ builder, surface_probe_sampler.h:120-223).

Layout. Nodes are u32[M][4] = (child_base, child_mask, probe_start,
probe_count). A branch has child_mask != 0: its present octants (bit o for
octant o, o = x | y << 1 | z << 2 with a bit set where position >
float32(center)) are stored contiguously from child_base in ascending octant
order. A leaf has child_mask == 0 and names the range [probe_start,
probe_start + probe_count) of the reordered probes. Numbering follows a
depth-first, octant-ordered walk in which a node's children are appended at
the moment it splits; leaves list their points in ascending input order.
The root cube is centred on the bounding box with half-extent
max(box) / 2 (at least 1e-5) grown by 1.0001; child centres are computed in
float64.

query_probe_indices restates SurfaceProbeLayout.query_probe_indices
(surface_probes.py:3016-3099): the probes of one instance within a radius,
optionally passing the hard normal gate.
"""

from __future__ import annotations

import numpy as np

SURFACE_PROBE_HARD_NORMAL_COSINE = 0.17364818

_OCTANT_SIGNS = np.array([[1.0 if o & 1 else -1.0, 1.0 if o & 2 else -1.0, 1.0 if o & 4 else -1.0]
                          for o in range(8)], dtype=np.float64)


def build_point_octree(positions, *, leaf_capacity: int = 8, max_depth: int = 16):
    """Returns (nodes u32[M, 4], order i64[N], root_center (x, y, z), root_extent)."""
    p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    if p.shape[0] == 0:
        raise ValueError("a point octree needs at least one position")
    leaf_capacity = int(leaf_capacity)
    max_depth = int(max_depth)
    lo = p.min(axis=0).astype(np.float64)
    hi = p.max(axis=0).astype(np.float64)
    center = (lo + hi) * 0.5
    extent = max(float(np.max(hi - lo)) * 0.5, 1e-5) * 1.0001

    nodes = [[0, 0, 0, 0]]
    order_parts: list[np.ndarray] = []
    placed = 0
    # Work items: (node index, point indices in ascending order, centre, half extent, depth).
    stack = [(0, np.arange(p.shape[0], dtype=np.int64), center, extent, 0)]
    while stack:
        node, idx, c, e, depth = stack.pop()
        if idx.size <= leaf_capacity or depth >= max_depth:
            nodes[node] = [0, 0, placed, int(idx.size)]
            order_parts.append(idx)
            placed += int(idx.size)
            continue
        above = p[idx] > c.astype(np.float32)
        octant = above[:, 0].astype(np.uint8) | (above[:, 1].astype(np.uint8) << 1) | (
            above[:, 2].astype(np.uint8) << 2)
        counts = np.bincount(octant, minlength=8)
        present = np.flatnonzero(counts)
        base = len(nodes)
        nodes.extend([0, 0, 0, 0] for _ in present)
        nodes[node] = [base, int(np.sum(1 << present)), 0, 0]
        grouped = idx[np.argsort(octant, kind="stable")]
        ends = np.cumsum(counts[present])
        starts = ends - counts[present]
        half = e * 0.5
        children = [(base + k, grouped[starts[k]:ends[k]], c + _OCTANT_SIGNS[o] * half, half, depth + 1)
                    for k, o in enumerate(present)]
        stack.extend(reversed(children))  # octant 0 is walked first
    order = np.concatenate(order_parts) if order_parts else np.zeros(0, np.int64)
    return (np.asarray(nodes, dtype=np.uint32), order.astype(np.int64),
            (float(center[0]), float(center[1]), float(center[2])), float(extent))


def _sphere_meets_cube(position, radius, center, extent) -> bool:
    d = np.maximum(np.abs(position - center) - extent, 0.0)
    return float(np.dot(d, d)) <= radius * radius


def query_probe_indices(layout, instance_index: int, position, radius: float | None = None, normal=None):
    """Probe indices of one instance within `radius` (default: its kernel
    radius) of `position`; with `normal`, only probes whose normal has a
    cosine of at least the hard gate with it. `layout` has nodes, probes and
    instance_infos (root_center, root_extent, node_offset, kernel_radius)."""
    info = layout.instance_infos[int(instance_index)]
    q = np.asarray(position, dtype=np.float64)
    r = info.kernel_radius if radius is None else max(float(radius), 0.0)
    qn = None if normal is None else np.asarray(normal, dtype=np.float64)
    found: list[int] = []
    stack = [(info.node_offset, np.asarray(info.root_center, dtype=np.float64), info.root_extent)]
    while stack:
        node, c, e = stack.pop()
        if not _sphere_meets_cube(q, r, c, e):
            continue
        child_base, mask, start, count = (int(v) for v in layout.nodes[node])
        if mask == 0:
            for k in range(start, start + count):
                d = layout.probes["position_radius"][k, :3].astype(np.float64) - q
                if float(np.dot(d, d)) > r * r:
                    continue
                if qn is not None and float(np.dot(qn, layout.probes["normal_side"][k, :3].astype(np.float64))) \
                        < SURFACE_PROBE_HARD_NORMAL_COSINE:
                    continue
                found.append(k)
            continue
        half = e * 0.5
        compact = 0
        for o in range(8):
            if not mask & (1 << o):
                continue
            cc = c + _OCTANT_SIGNS[o] * half
            if _sphere_meets_cube(q, r, cc, half):
                stack.append((child_base + compact, cc, half))
            compact += 1
    return np.asarray(found, dtype=np.int64)
