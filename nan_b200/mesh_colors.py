"""Mesh Colors layout (host side): mesh_colors.py:24-337 of the reference.

Each triangle gets a power-of-two lattice resolution R from its longest
world-space edge, R = min(nextpow2(max(min_res, ceil(edge * texels_per_unit))),
max_res), and (R+1)(R+2)/2 texels. Instances are laid out front range first,
then (for double-sided materials) a back range of the same size. When the
running total would exceed the texel budget, later triangles are halved
greedily toward min_res (mesh_colors.py:231-251), and a layout that cannot
fit raises ValueError("Mesh Colors texel budget exceeded ...").
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

MESH_COLORS_PAYLOAD_SIZE = 16
MESH_COLORS_INVALID_OFFSET = 0xFFFFFFFF
MESH_COLORS_SIDE_FLAG_DOUBLE_SIDED = 1 << 0


def colors_per_patch(resolution: int) -> int:
    resolution = int(resolution)
    if resolution < 1:
        raise ValueError("resolution must be positive")
    return (resolution + 1) * (resolution + 2) // 2


def address_to_ij(address: int, resolution: int) -> tuple[int, int]:
    """Triangle-local linear address -> lattice (i, j) (closed form + fix-up)."""
    address, resolution = int(address), int(resolution)
    if address < 0 or address >= colors_per_patch(resolution):
        raise ValueError("address is outside the triangle patch")
    b = 2 * resolution + 3
    i = int((b - math.sqrt(b * b - 8 * address)) * 0.5)
    cumulative = i * (resolution + 1) - i * (i - 1) // 2
    while cumulative > address:
        i -= 1
        cumulative = i * (resolution + 1) - i * (i - 1) // 2
    while i < resolution:
        nxt = (i + 1) * (resolution + 1) - (i + 1) * i // 2
        if nxt > address:
            break
        i += 1
        cumulative = nxt
    return i, address - cumulative


def ij_to_address(i: int, j: int, resolution: int) -> int:
    i, j, resolution = int(i), int(j), int(resolution)
    if i < 0 or i > resolution or j < 0 or j > resolution - i:
        raise ValueError("(i, j) is outside the triangle patch")
    return i * (resolution + 1) - i * (i - 1) // 2 + j


def barycentric_at(i: int, j: int, resolution: int) -> tuple[float, float, float]:
    if resolution <= 0:
        raise ValueError("resolution must be positive")
    u = float(i) / float(resolution)
    v = float(j) / float(resolution)
    return u, v, 1.0 - u - v


def next_power_of_two(value: int) -> int:
    value = max(1, int(value))
    return 1 << (value - 1).bit_length()


def previous_power_of_two(value: int) -> int:
    value = max(1, int(value))
    return 1 << (value.bit_length() - 1)


@dataclass(frozen=True)
class MeshColorsFaceInfo:
    address: int
    resolution: int


@dataclass(frozen=True)
class MeshColorsInstanceInfo:
    face_offset: int
    face_count: int
    texel_offset: int
    texel_count: int


@dataclass(frozen=True)
class MeshColorsSideInfo:
    back_texel_offset: int
    flags: int

    @property
    def is_double_sided(self) -> bool:
        return bool(self.flags & MESH_COLORS_SIDE_FLAG_DOUBLE_SIDED)


def _patch(r: np.ndarray) -> np.ndarray:
    r = r.astype(np.int64)
    return (r + 1) * (r + 2) // 2


def _wanted_resolutions(scene_node, texels_per_unit: float, min_resolution: int, max_resolution: int,
                        chunk_triangles: int = 1 << 20) -> list:
    """Per instance, each triangle's patch resolution before the texel
    budget: the power of two at or above its longest world-space edge x
    texels_per_unit, clamped to [min_resolution, max_resolution]. The
    instances of one mesh are transformed together (in chunks of about
    chunk_triangles triangles), each with the arithmetic of its own
    transform alone."""
    out = [None] * len(scene_node.instances)
    groups: dict = {}
    for i, (mesh_id, _, _) in enumerate(scene_node.instances):
        groups.setdefault(mesh_id, []).append(i)
    for mesh_id, members in groups.items():
        mesh = scene_node.meshes[mesh_id]
        p = mesh.vertices[:, 0:3].astype(np.float32)
        idx = mesh.indices.astype(np.int64)
        step = max(1, chunk_triangles // max(mesh.triangle_count, 1))
        for c in range(0, len(members), step):
            part = members[c:c + step]
            m = np.stack([np.asarray(scene_node.transforms[scene_node.instances[i][2]], dtype=np.float32)
                          for i in part])
            world = (p @ m[:, :3, :3].transpose(0, 2, 1) + m[:, None, :3, 3]).astype(np.float32).astype(np.float64)
            tri = world[:, idx]  # [g, T, 3, 3]
            e = np.stack([
                np.linalg.norm(tri[:, :, 1] - tri[:, :, 0], axis=2),
                np.linalg.norm(tri[:, :, 2] - tri[:, :, 1], axis=2),
                np.linalg.norm(tri[:, :, 0] - tri[:, :, 2], axis=2),
            ], axis=2).max(axis=2)
            want = np.maximum(min_resolution, np.ceil(e * texels_per_unit)).astype(np.int64)
            want = np.maximum(want, 1)
            res = np.left_shift(1, np.ceil(np.log2(want)).astype(np.int64))
            res = np.where(res < want, res * 2, res)  # guard log2 rounding
            res = np.minimum(res, max_resolution)
            for j, i in enumerate(part):
                out[i] = res[j]
    return out


class MeshColorsLayout:
    """Layout arrays: face_infos u32[F,2], instance_infos u32[I,4], side_infos u32[I,2]."""

    def __init__(self, face_infos, instance_infos, side_infos, total_surface_texels, total_payload_count,
                 texels_per_unit, min_resolution, max_resolution):
        self.face_array = np.ascontiguousarray(face_infos, dtype=np.uint32).reshape(-1, 2)
        self.instance_array = np.ascontiguousarray(instance_infos, dtype=np.uint32).reshape(-1, 4)
        self.side_array = np.ascontiguousarray(side_infos, dtype=np.uint32).reshape(-1, 2)
        self.total_surface_texels = int(total_surface_texels)
        self.total_payload_count = int(total_payload_count)
        self.texels_per_unit = float(texels_per_unit)
        self.min_resolution = int(min_resolution)
        self.max_resolution = int(max_resolution)

    @property
    def total_texel_count(self) -> int:
        return self.total_surface_texels

    @property
    def face_infos(self) -> tuple:
        return tuple(MeshColorsFaceInfo(int(a), int(r)) for a, r in self.face_array)

    @property
    def instance_infos(self) -> tuple:
        return tuple(MeshColorsInstanceInfo(*(int(x) for x in row)) for row in self.instance_array)

    @property
    def side_infos(self) -> tuple:
        return tuple(MeshColorsSideInfo(int(a), int(f)) for a, f in self.side_array)

    @property
    def surface_prefix(self) -> np.ndarray:
        """Exclusive prefix of the instances' surface texel counts, u32[I+1]."""
        counts = self.instance_array[:, 3].astype(np.int64)
        return np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)

    @classmethod
    def build(cls, scene_node, *, texels_per_unit: float = 16.0, min_resolution: int = 4,
              max_resolution: int = 64, max_total_texels: int = 16_777_216) -> "MeshColorsLayout":
        texels_per_unit = max(float(texels_per_unit), 1e-6)
        min_resolution = next_power_of_two(max(1, int(min_resolution)))
        max_resolution = previous_power_of_two(max(1, int(max_resolution)))
        if min_resolution > max_resolution:
            raise ValueError(
                "Mesh Colors min_resolution must not exceed max_resolution after power-of-two normalization"
            )
        max_total_texels = max(1, int(max_total_texels))
        faces, instances, sides = [], [], []
        face_count = 0
        total_surface = 0
        total_payload = 0
        wanted = _wanted_resolutions(scene_node, texels_per_unit, min_resolution, max_resolution)
        n_inst = len(scene_node.instances)
        double = np.array([bool(getattr(scene_node.materials[mat], "double_sided", False))
                           for _, mat, _ in scene_node.instances], dtype=bool)
        mult_all = np.where(double, 2, 1).astype(np.int64)
        # the instances before the first one that would exceed the budget at
        # its wanted resolutions are laid out in one pass
        tri_n = np.array([w.shape[0] for w in wanted], np.int64)
        flat_res = np.concatenate(wanted) if n_inst else np.zeros(0, np.int64)
        flat_patch = _patch(flat_res)
        tri_start = np.concatenate([[0], np.cumsum(tri_n)])
        patch_cum = np.concatenate([[0], np.cumsum(flat_patch)])
        local_totals = patch_cum[tri_start[1:]] - patch_cum[tri_start[:-1]]
        payload_after = np.cumsum(local_totals * mult_all)
        over = np.flatnonzero((tri_n > 0) & (payload_after > max_total_texels))
        k0 = int(over[0]) if over.size else n_inst
        if k0:
            e = int(tri_start[k0])
            owner = np.repeat(np.arange(k0), tri_n[:k0])
            addresses = (patch_cum[1:e + 1] - patch_cum[tri_start[owner]] - flat_patch[:e]).astype(np.uint32)
            faces.append(np.stack([addresses, flat_res[:e].astype(np.uint32)], axis=1))
            face_off = tri_start[:k0]
            pay_off = np.concatenate([[0], payload_after[:k0 - 1]]) if k0 > 1 else np.zeros(1, np.int64)
            instances.extend(zip(face_off.tolist(), tri_n[:k0].tolist(), pay_off.tolist(),
                                 local_totals[:k0].tolist()))
            back = np.where(double[:k0], pay_off + local_totals[:k0], MESH_COLORS_INVALID_OFFSET)
            flag = np.where(double[:k0], MESH_COLORS_SIDE_FLAG_DOUBLE_SIDED, 0)
            sides.extend(zip(back.tolist(), flag.tolist()))
            face_count = e
            total_surface = int(local_totals[:k0].sum())
            total_payload = int(payload_after[k0 - 1])
        for inst_k in range(k0, n_inst):
            mesh = scene_node.meshes[scene_node.instances[inst_k][0]]
            double_sided = bool(double[inst_k])
            mult = 2 if double_sided else 1
            res = wanted[inst_k]
            patch = _patch(res)
            cum = np.cumsum(patch)
            face_offset = face_count
            if mesh.triangle_count and total_payload + int(cum[-1]) * mult > max_total_texels:
                res = res.copy()
                local = 0
                for k in range(mesh.triangle_count):
                    r = int(res[k])
                    pt = colors_per_patch(r)
                    if total_payload + (local + pt) * mult > max_total_texels:
                        cand = r
                        fitted = False
                        while cand > min_resolution:
                            cand //= 2
                            pt = colors_per_patch(cand)
                            if total_payload + (local + pt) * mult <= max_total_texels:
                                r = cand
                                fitted = True
                                break
                        if not fitted:
                            raise ValueError(
                                "Mesh Colors texel budget exceeded; lower --texture-space-texels-per-unit "
                                "or --texture-space-min-resolution, or increase --texture-space-max-texels"
                            )
                    res[k] = r
                    local += pt
                patch = _patch(res)
                cum = np.cumsum(patch)
            addresses = (cum - patch).astype(np.uint32)
            faces.append(np.stack([addresses, res.astype(np.uint32)], axis=1))
            face_count += faces[-1].shape[0]
            local_total = int(cum[-1]) if mesh.triangle_count else 0
            instances.append((face_offset, mesh.triangle_count, total_payload, local_total))
            back = total_payload + local_total if double_sided else MESH_COLORS_INVALID_OFFSET
            sides.append((back, MESH_COLORS_SIDE_FLAG_DOUBLE_SIDED if double_sided else 0))
            total_surface += local_total
            total_payload += local_total * mult
        if total_surface == 0:
            raise ValueError("Texture-space rendering requires at least one triangle")
        face_array = np.concatenate(faces, axis=0) if faces else np.zeros((0, 2), np.uint32)
        return cls(face_array, np.asarray(instances, dtype=np.uint32), np.asarray(sides, dtype=np.uint32),
                   total_surface, total_payload, texels_per_unit, min_resolution, max_resolution)

    def create_gpu_buffers(self, device):
        """(face_infos, instance_infos, side_infos, surface_prefix) as int32 CUDA tensors."""
        import torch

        td = device.torch_device if hasattr(device, "torch_device") else device
        def up(a):
            return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(td)
        return up(self.face_array), up(self.instance_array), up(self.side_array), up(self.surface_prefix)

    def units(self) -> np.ndarray:
        """Every (instance, instance-local texel) pair in surface-texel order, u32[N,2]."""
        counts = self.instance_array[:, 3].astype(np.int64)
        inst = np.repeat(np.arange(len(counts), dtype=np.uint32), counts)
        local = np.arange(int(counts.sum()), dtype=np.int64) - np.repeat(self.surface_prefix[:-1].astype(np.int64),
                                                                         counts)
        return np.stack([inst, local.astype(np.uint32)], axis=1)


# Edge adjacency of a triangle mesh (mesh_colors_adjacency.py:164-246 of the
# reference): edge e of a face runs from vertex e to vertex (e + 1) % 3; a
# manifold edge (used by exactly two faces) links each face to the other as
# (adjacent face << 3) | adjacent edge | flip << 2, where flip means the two
# faces traverse the edge in opposite directions; other edges stay ~0.
ADJACENCY_INVALID = 0xFFFFFFFF


def build_triangle_adjacency(indices) -> np.ndarray:
    """u32[F][4]: packed adjacency of edges 0..2, then ~0."""
    tri = np.asarray(indices, dtype=np.int64).reshape(-1, 3)
    n = tri.shape[0]
    out = np.full((n, 4), ADJACENCY_INVALID, dtype=np.uint32)
    if n == 0:
        return out
    good = (tri[:, 0] != tri[:, 1]) & (tri[:, 1] != tri[:, 2]) & (tri[:, 0] != tri[:, 2])
    f = np.repeat(np.arange(n), 3)
    e = np.tile(np.arange(3), n)
    a = tri[f, e]
    b = tri[f, (e + 1) % 3]
    keep = good[f]
    f, e, a, b = f[keep], e[keep], a[keep], b[keep]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    order = np.lexsort((e, f, hi, lo))  # by edge key, then in insertion order (face, edge)
    f, e, a, b, lo, hi = f[order], e[order], a[order], b[order], lo[order], hi[order]
    starts = np.flatnonzero(np.r_[True, (lo[1:] != lo[:-1]) | (hi[1:] != hi[:-1])])
    sizes = np.diff(np.r_[starts, lo.size])
    pair = starts[sizes == 2]
    first, second = pair, pair + 1
    ok = f[first] != f[second]
    first, second = first[ok], second[ok]
    flip = (a[first] == b[second]) & (b[first] == a[second])
    fl = np.where(flip, 4, 0).astype(np.int64)
    out[f[first], e[first]] = ((f[second] << 3) | e[second] | fl).astype(np.uint32)
    out[f[second], e[second]] = ((f[first] << 3) | e[first] | fl).astype(np.uint32)
    return out


def layout_adjacency(scene_node) -> np.ndarray:
    """u32[F][4] for every face of the layout (instances in order, mesh-local
    adjacent face indices), as the filter reads it."""
    per_mesh = {}
    rows = []
    for mesh_id, _, _ in scene_node.instances:
        if mesh_id not in per_mesh:
            per_mesh[mesh_id] = build_triangle_adjacency(scene_node.meshes[mesh_id].indices)
        rows.append(per_mesh[mesh_id])
    return np.concatenate(rows) if rows else np.zeros((0, 4), np.uint32)


def layout_face_normals(scene_node) -> np.ndarray:
    """f32[F][4]: unit world-space face normals (0 for degenerate faces)."""
    rows = []
    for mesh_id, _, transform_id in scene_node.instances:
        mesh = scene_node.meshes[mesh_id]
        m = np.asarray(scene_node.transforms[transform_id], dtype=np.float64)
        p = mesh.vertices[:, 0:3].astype(np.float64) @ m[:3, :3].T + m[:3, 3]
        tri = p[mesh.indices.astype(np.int64)]
        nrm = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
        length = np.linalg.norm(nrm, axis=1, keepdims=True)
        nrm = np.where(length > 1e-20, nrm / np.maximum(length, 1e-300), 0.0)
        r = np.zeros((tri.shape[0], 4), np.float32)
        r[:, :3] = nrm
        rows.append(r)
    return np.concatenate(rows) if rows else np.zeros((0, 4), np.float32)
