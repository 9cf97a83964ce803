"""Host-side scene description: meshes, materials, transforms, instances.

Mirrors the parts of the reference's SceneNode/Mesh/Material/Transform that
feed the path-integration kernels (scene_node.py, mesh.py:6-189,
material.py, transform.py:12-16). Asset loading (glTF/OBJ) is not part of
this package; scenes come from the seeded generators in nan_b200.scenes.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MATERIAL_FLAG_DOUBLE_SIDED = 1 << 0
INSTANCE_FLAG_ODD_NEGATIVE_TRANSFORM = 1 << 0


@dataclass
class Mesh:
    """vertices f32[V,8] (position, normal, uv) and indices u32[T,3]."""

    vertices: np.ndarray
    indices: np.ndarray

    def __post_init__(self):
        self.vertices = np.ascontiguousarray(self.vertices, dtype=np.float32)
        self.indices = np.ascontiguousarray(self.indices, dtype=np.uint32)
        if self.vertices.ndim != 2 or self.vertices.shape[1] != 8:
            raise ValueError("mesh vertices must be float32 [V, 8]")
        if self.indices.ndim != 2 or self.indices.shape[1] != 3:
            raise ValueError("mesh indices must be uint32 [T, 3]")

    @property
    def vertex_count(self) -> int:
        return int(self.vertices.shape[0])

    @property
    def triangle_count(self) -> int:
        return int(self.indices.shape[0])

    @property
    def index_count(self) -> int:
        return 3 * self.triangle_count

    # Geometry factories with the reference's vertex order and winding
    # (mesh.py:65-189), used to rebuild its demo scene.
    @classmethod
    def quad(cls, size=(1.0, 1.0)) -> "Mesh":
        v = np.array(
            [[-0.5, 0, -0.5, 0, 1, 0, 0, 0], [0.5, 0, -0.5, 0, 1, 0, 1, 0],
             [-0.5, 0, 0.5, 0, 1, 0, 0, 1], [0.5, 0, 0.5, 0, 1, 0, 1, 1]], dtype=np.float32)
        v[:, 0] *= size[0]
        v[:, 2] *= size[1]
        return cls(v, np.array([[2, 1, 0], [1, 2, 3]], dtype=np.uint32))

    @classmethod
    def quad_yz(cls, size=(1.0, 1.0), face_positive_x: bool = True) -> "Mesh":
        nx = 1.0 if face_positive_x else -1.0
        v = np.array(
            [[0, -0.5, -0.5, nx, 0, 0, 0, 0], [0, 0.5, -0.5, nx, 0, 0, 1, 0],
             [0, -0.5, 0.5, nx, 0, 0, 0, 1], [0, 0.5, 0.5, nx, 0, 0, 1, 1]], dtype=np.float32)
        v[:, 1] *= size[0]
        v[:, 2] *= size[1]
        idx = [[0, 1, 2], [3, 2, 1]] if face_positive_x else [[2, 1, 0], [1, 2, 3]]
        return cls(v, np.array(idx, dtype=np.uint32))

    @classmethod
    def quad_xy(cls, size=(1.0, 1.0), face_positive_z: bool = True) -> "Mesh":
        nz = 1.0 if face_positive_z else -1.0
        v = np.array(
            [[-0.5, -0.5, 0, 0, 0, nz, 0, 0], [0.5, -0.5, 0, 0, 0, nz, 1, 0],
             [-0.5, 0.5, 0, 0, 0, nz, 0, 1], [0.5, 0.5, 0, 0, 0, nz, 1, 1]], dtype=np.float32)
        v[:, 0] *= size[0]
        v[:, 1] *= size[1]
        idx = [[0, 1, 2], [3, 2, 1]] if face_positive_z else [[2, 1, 0], [1, 2, 3]]
        return cls(v, np.array(idx, dtype=np.uint32))

    @classmethod
    def cube(cls, size=(1.0, 1.0, 1.0)) -> "Mesh":
        """Box with outward faces, 24 vertices and 12 triangles, in the
        reference's vertex order and winding (mesh.py:131-189): faces -y, +y,
        -z, +z, -x, +x; face corners (n + a + b, n + a - b, n - a - b,
        n - a + b) / 2 with uvs (0,0), (1,0), (1,1), (0,1); triangles
        (0, 2, 1) and (0, 3, 2) of each face."""
        faces = [  # (normal n, edge a, edge b)
            ((0, -1, 0), (-1, 0, 0), (0, 0, -1)),
            ((0, 1, 0), (-1, 0, 0), (0, 0, 1)),
            ((0, 0, -1), (-1, 0, 0), (0, 1, 0)),
            ((0, 0, 1), (1, 0, 0), (0, 1, 0)),
            ((-1, 0, 0), (0, 0, 1), (0, 1, 0)),
            ((1, 0, 0), (0, 0, -1), (0, 1, 0)),
        ]
        corners = ((1, 1), (1, -1), (-1, -1), (-1, 1))
        uvs = ((0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0))
        verts, idx = [], []
        for n, a, b in faces:
            n, a, b = np.array(n, float), np.array(a, float), np.array(b, float)
            base = len(verts)
            for (sa, sb), uv in zip(corners, uvs):
                verts.append([*(0.5 * (n + sa * a + sb * b)), *n, *uv])
            idx += [[base, base + 2, base + 1], [base, base + 3, base + 2]]
        v = np.array(verts, dtype=np.float32)
        v[:, 0:3] *= np.asarray(size, dtype=np.float32)
        return cls(v, np.array(idx, dtype=np.uint32))


@dataclass
class Material:
    """Opaque Lambert material (material.py): base color, emission, sidedness."""

    base_color: tuple = (0.5, 0.5, 0.5)
    emissive: tuple = (0.0, 0.0, 0.0)
    double_sided: bool = False

    @property
    def flags(self) -> int:
        return MATERIAL_FLAG_DOUBLE_SIDED if self.double_sided else 0

    def pack(self) -> np.ndarray:
        """f32[8]: base_color.rgb, flags (u32 bits), emissive.rgb, pad."""
        rec = np.zeros(8, dtype=np.float32)
        rec[0:3] = self.base_color
        rec[3:4] = np.array([self.flags], dtype=np.uint32).view(np.float32)
        rec[4:7] = self.emissive
        return rec


def rotation_y(angle: float) -> np.ndarray:
    c, s = np.cos(angle), np.sin(angle)
    return np.array([[c, 0, s, 0], [0, 1, 0, 0], [-s, 0, c, 0], [0, 0, 0, 1]], dtype=np.float64)


def rotation_x(angle: float) -> np.ndarray:
    c, s = np.cos(angle), np.sin(angle)
    return np.array([[1, 0, 0, 0], [0, c, -s, 0], [0, s, c, 0], [0, 0, 0, 1]], dtype=np.float64)


def rotation_z(angle: float) -> np.ndarray:
    c, s = np.cos(angle), np.sin(angle)
    return np.array([[c, -s, 0, 0], [s, c, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]], dtype=np.float64)


def make_transform(translation=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0), scaling=(1.0, 1.0, 1.0)) -> np.ndarray:
    """T * R * S with R = Rx * Ry * Rz (transform.py:12-16), float32 [4,4]."""
    t = np.eye(4)
    t[0:3, 3] = translation
    r = rotation_x(rotation[0]) @ rotation_y(rotation[1]) @ rotation_z(rotation[2])
    s = np.diag([scaling[0], scaling[1], scaling[2], 1.0])
    return (t @ r @ s).astype(np.float32)


@dataclass
class SceneNode:
    meshes: list = field(default_factory=list)
    materials: list = field(default_factory=list)
    transforms: list = field(default_factory=list)
    instances: list = field(default_factory=list)  # (mesh_id, material_id, transform_id)
    camera: object = None
    lighting: object = None
    name: str = "scene"

    def add_mesh(self, mesh: Mesh) -> int:
        self.meshes.append(mesh)
        return len(self.meshes) - 1

    def add_material(self, material: Material) -> int:
        self.materials.append(material)
        return len(self.materials) - 1

    def add_transform(self, matrix: np.ndarray) -> int:
        self.transforms.append(np.asarray(matrix, dtype=np.float32).reshape(4, 4))
        return len(self.transforms) - 1

    def add_instance(self, mesh_id: int, material_id: int, transform_id: int) -> int:
        self.instances.append((int(mesh_id), int(material_id), int(transform_id)))
        return len(self.instances) - 1

    @property
    def triangle_count(self) -> int:
        return sum(self.meshes[m].triangle_count for m, _, _ in self.instances)

    def pack(self) -> dict:
        """The reference's GPU record layouts (scene.py:84-108, 330-436)."""
        vertices = np.concatenate([m.vertices for m in self.meshes], axis=0)
        indices = np.concatenate([m.indices for m in self.meshes], axis=0)
        mesh_descs = np.zeros((len(self.meshes), 4), dtype=np.uint32)
        v_off = i_off = 0
        for k, m in enumerate(self.meshes):
            mesh_descs[k] = (m.vertex_count, m.index_count, v_off, i_off)
            v_off += m.vertex_count
            i_off += m.index_count
        instance_descs = np.zeros((len(self.instances), 4), dtype=np.uint32)
        stacked = np.stack(self.transforms).astype(np.float64).reshape(-1, 4, 4)
        if self.instances:
            ids = np.asarray(self.instances, dtype=np.int64).reshape(-1, 3)
            m = stacked[ids[:, 2], :3, :3]
            det = (np.cross(m[:, 0], m[:, 1]) * m[:, 2]).sum(axis=1)
            # the sign decides; near zero it is taken as np.dot forms it
            for k in np.flatnonzero(np.abs(det) <= 1e-9):
                det[k] = np.dot(np.cross(m[k, 0], m[k, 1]), m[k, 2])
            instance_descs[:, :3] = ids
            instance_descs[:, 3] = np.where(det <= 0, INSTANCE_FLAG_ODD_NEGATIVE_TRANSFORM, 0)
        transforms = stacked.astype(np.float32).reshape(-1, 16)
        inverse_transposes = np.linalg.inv(stacked).transpose(0, 2, 1).astype(np.float32).reshape(-1, 16)
        materials = np.stack([m.pack() for m in self.materials]).astype(np.float32)
        return {
            "vertices": np.ascontiguousarray(vertices, dtype=np.float32),
            "indices": np.ascontiguousarray(indices, dtype=np.uint32),
            "mesh_descs": mesh_descs,
            "instance_descs": instance_descs,
            "transforms": np.ascontiguousarray(transforms),
            "inverse_transposes": np.ascontiguousarray(inverse_transposes),
            "materials": np.ascontiguousarray(materials),
        }
