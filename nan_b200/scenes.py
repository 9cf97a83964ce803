"""Seeded synthetic scenes for the path-integration workloads.

No asset or dataset is involved: every scene is generated from
``numpy.random.default_rng(seed)`` with the shapes, sizes and value
distributions of the workload it stands for.

* ``cornell_box()``      -- 5 walls of a 2x2x2 box (10 triangles), two
  axis-aligned boxes 0.6x0.6x0.6 and 0.6x1.2x0.6 (24), a 0.5x0.5 ceiling
  light with emission (17, 12, 4) (2): 36 triangles; white 0.73, red
  (0.63, 0.065, 0.05), green (0.14, 0.45, 0.09); lit by the quad only.
* ``reference_demo()``   -- the reference's SceneNode.demo() Cornell box
  (scene_node.py:721-831): used to cross-check layout numbers its tests pin.
* ``terrain_boxes()``    -- displaced-grid terrain (heights = 2 x smoothed
  noise) plus 500 boxes with sides U[0.2, 3] and random yaw; albedo
  U[0.1, 0.9]; sun at 45 deg elevation with irradiance 3, sky 0.5. The
  default 313x313 grid gives 194,688 + 6,000 = 200,688 triangles.
* ``city()``             -- 20k boxes (one tessellated box mesh, instanced)
  with heights log-normal (mu 2, sigma 0.7) on a 2 km grid plus a
  tessellated ground plane: about 4.16 M triangles; sun at 30 deg and sky.
* ``batch_scenes()``     -- many terrain_boxes scenes with triangle counts
  log-uniform in [1e3, 5e5] and a site count U{512..20480} each (the
  multi-scene probe workload).
"""

from __future__ import annotations

import math

import numpy as np

from .camera import Camera
from .scene import Lighting
from .scene_node import Material, Mesh, SceneNode, make_transform
from .surface_probe_resources import (SURFACE_PROBE_DTYPE, SURFACE_PROBE_FLAG_BACK_SIDE,
                                      SURFACE_PROBE_INSTANCE_DTYPE, SURFACE_PROBE_INSTANCE_SHIFT)


def _camera(position, target, fov, width=256, height=256) -> Camera:
    cam = Camera()
    cam.position = np.asarray(position, dtype=np.float32)
    cam.target = np.asarray(target, dtype=np.float32)
    cam.fov = float(fov)
    cam.width, cam.height = width, height
    cam.recompute()
    return cam


def cornell_box(width: int = 256, height: int = 256) -> SceneNode:
    s = SceneNode(name="cornell_box_36")
    white = s.add_material(Material((0.73, 0.73, 0.73), double_sided=True))
    red = s.add_material(Material((0.63, 0.065, 0.05), double_sided=True))
    green = s.add_material(Material((0.14, 0.45, 0.09), double_sided=True))
    box_white = s.add_material(Material((0.73, 0.73, 0.73)))
    light = s.add_material(Material((0.0, 0.0, 0.0), emissive=(17.0, 12.0, 4.0)))
    floor = s.add_mesh(Mesh.quad((2.0, 2.0)))
    back = s.add_mesh(Mesh.quad_xy((2.0, 2.0), face_positive_z=True))
    left = s.add_mesh(Mesh.quad_yz((2.0, 2.0), face_positive_x=True))
    right = s.add_mesh(Mesh.quad_yz((2.0, 2.0), face_positive_x=False))
    s.add_instance(floor, white, s.add_transform(make_transform((0, 0, 0))))
    s.add_instance(floor, white, s.add_transform(make_transform((0, 2, 0), (math.pi, 0, 0))))
    s.add_instance(back, white, s.add_transform(make_transform((0, 1, -1))))
    s.add_instance(left, red, s.add_transform(make_transform((-1, 1, 0))))
    s.add_instance(right, green, s.add_transform(make_transform((1, 1, 0))))
    short_box = s.add_mesh(Mesh.cube((0.6, 0.6, 0.6)))
    tall_box = s.add_mesh(Mesh.cube((0.6, 1.2, 0.6)))
    s.add_instance(tall_box, box_white, s.add_transform(make_transform((-0.35, 0.6, -0.3))))
    s.add_instance(short_box, box_white, s.add_transform(make_transform((0.35, 0.3, 0.3))))
    lq = s.add_mesh(Mesh.quad((0.5, 0.5)))
    s.add_instance(lq, light, s.add_transform(make_transform((0, 1.99, 0), (math.pi, 0, 0))))
    s.camera = _camera((0.0, 1.0, 3.9), (0.0, 1.0, 0.0), 40.0, width, height)
    s.lighting = Lighting(sun_intensity=0.0, sky_radiance=(0.0, 0.0, 0.0), sun_disk=False)
    return s


def reference_demo() -> SceneNode:
    """The reference's demo Cornell box (scene_node.py:721-831)."""
    s = SceneNode(name="reference_demo")
    white_wall = s.add_material(Material((0.73, 0.73, 0.73), double_sided=True))
    red_wall = s.add_material(Material((0.65, 0.05, 0.05), double_sided=True))
    green_wall = s.add_material(Material((0.12, 0.45, 0.15), double_sided=True))
    white_box = s.add_material(Material((0.73, 0.73, 0.73)))
    light = s.add_material(Material((1.0, 1.0, 1.0), emissive=(15.0, 15.0, 15.0)))
    quad = s.add_mesh(Mesh.quad((2, 2)))
    back = s.add_mesh(Mesh.quad_xy((2, 2), face_positive_z=True))
    left = s.add_mesh(Mesh.quad_yz((2, 2), face_positive_x=True))
    right = s.add_mesh(Mesh.quad_yz((2, 2), face_positive_x=False))
    s.add_instance(quad, white_wall, s.add_transform(make_transform((0, 0, 0))))
    s.add_instance(quad, white_wall, s.add_transform(make_transform((0, 2, 0), (math.pi, 0, 0))))
    s.add_instance(back, white_wall, s.add_transform(make_transform((0, 1, -1))))
    s.add_instance(left, red_wall, s.add_transform(make_transform((-1, 1, 0))))
    s.add_instance(right, green_wall, s.add_transform(make_transform((1, 1, 0))))
    lq = s.add_mesh(Mesh.quad((0.4, 0.4)))
    s.add_instance(lq, light, s.add_transform(make_transform((0, 1.99, 0), (math.pi, 0, 0))))
    tall = s.add_mesh(Mesh.cube((0.5, 1.2, 0.5)))
    s.add_instance(tall, white_box, s.add_transform(make_transform((-0.35, 0.6, -0.3), (0, 18, 0))))
    short = s.add_mesh(Mesh.cube((0.5, 0.6, 0.5)))
    s.add_instance(short, white_box, s.add_transform(make_transform((0.35, 0.3, 0.3), (0, -18, 0))))
    s.camera = _camera((0.0, 1.0, 2.95), (0.0, 1.0, 0.0), 60.0)
    s.lighting = Lighting()
    return s


def _smoothed_noise(rng: np.random.Generator, n: int, sigma_cells: float) -> np.ndarray:
    """White noise blurred by a Gaussian (FFT), scaled to [-1, 1]."""
    white = rng.standard_normal((n, n))
    k = np.fft.fftfreq(n)
    g = np.exp(-2.0 * (math.pi * sigma_cells) ** 2 * (k[:, None] ** 2 + k[None, :] ** 2))
    smooth = np.real(np.fft.ifft2(np.fft.fft2(white) * g))
    smooth -= smooth.mean()
    return smooth / max(np.abs(smooth).max(), 1e-12)


def grid_mesh(heights: np.ndarray, cell: float) -> Mesh:
    """Triangulated height field centred on the origin, normals from the grid."""
    n = heights.shape[0]
    half = 0.5 * cell * (n - 1)
    xs = np.arange(n, dtype=np.float64) * cell - half
    gx, gz = np.meshgrid(xs, xs, indexing="xy")
    h = heights.astype(np.float64)
    dhdx = np.gradient(h, cell, axis=1)
    dhdz = np.gradient(h, cell, axis=0)
    nrm = np.stack([-dhdx, np.ones_like(h), -dhdz], axis=-1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    v = np.zeros((n * n, 8), dtype=np.float32)
    v[:, 0] = gx.reshape(-1)
    v[:, 1] = h.reshape(-1)
    v[:, 2] = gz.reshape(-1)
    v[:, 3:6] = nrm.reshape(-1, 3)
    v[:, 6] = (gx.reshape(-1) + half) / (2 * half)
    v[:, 7] = (gz.reshape(-1) + half) / (2 * half)
    i = np.arange(n - 1)
    a = (i[:, None] * n + i[None, :]).reshape(-1)  # row z, col x
    b, c, d = a + 1, a + n, a + n + 1
    # counter-clockwise seen from +y: (a, c, b) and (b, c, d)
    tris = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)], axis=0)
    return Mesh(v, tris.astype(np.uint32))


def _height_at(heights: np.ndarray, cell: float, x: float, z: float) -> float:
    n = heights.shape[0]
    half = 0.5 * cell * (n - 1)
    fx = np.clip((x + half) / cell, 0, n - 1.001)
    fz = np.clip((z + half) / cell, 0, n - 1.001)
    ix, iz = int(fx), int(fz)
    tx, tz = fx - ix, fz - iz
    h00, h01 = heights[iz, ix], heights[iz, ix + 1]
    h10, h11 = heights[iz + 1, ix], heights[iz + 1, ix + 1]
    return float((h00 * (1 - tx) + h01 * tx) * (1 - tz) + (h10 * (1 - tx) + h11 * tx) * tz)


def terrain_boxes(seed: int = 1, grid: int = 313, cell: float = 0.15, boxes: int = 500,
                  amplitude: float = 2.0, noise_sigma_cells: float = 12.0) -> SceneNode:
    rng = np.random.default_rng(seed)
    s = SceneNode(name=f"terrain{grid}x{grid}_boxes{boxes}_seed{seed}")
    heights = amplitude * _smoothed_noise(rng, grid, noise_sigma_cells)
    terrain = s.add_mesh(grid_mesh(heights, cell))
    terrain_mat = s.add_material(Material(tuple(rng.uniform(0.1, 0.9, 3))))
    s.add_instance(terrain, terrain_mat, s.add_transform(np.eye(4, dtype=np.float32)))
    cube = s.add_mesh(Mesh.cube((1.0, 1.0, 1.0)))
    half = 0.5 * cell * (grid - 1)
    for _ in range(boxes):
        size = rng.uniform(0.2, 3.0, 3)
        yaw = rng.uniform(0.0, 2.0 * math.pi)
        x, z = rng.uniform(-half * 0.95, half * 0.95, 2)
        y = _height_at(heights, cell, x, z) + 0.5 * size[1] - 0.1 * size[1]
        mat = s.add_material(Material(tuple(rng.uniform(0.1, 0.9, 3))))
        s.add_instance(cube, mat, s.add_transform(make_transform((x, y, z), (0.0, yaw, 0.0), size)))
    extent = 2 * half
    s.camera = _camera((0.0, amplitude + 0.25 * extent, 0.6 * extent), (0.0, 0.0, 0.0), 60.0)
    s.lighting = Lighting.sun_elevation(45.0, azimuth_deg=30.0, irradiance=3.0, sky=0.5)
    s.terrain_cell = cell
    return s


def tessellated_box(n: int) -> Mesh:
    """Unit box (centred, outward faces) with every face split into n x n
    quads: 12 n^2 triangles."""
    faces = [((0, -1, 0), (0, 0, 1), (1, 0, 0)), ((0, 1, 0), (1, 0, 0), (0, 0, 1)),
             ((0, 0, -1), (1, 0, 0), (0, 1, 0)), ((0, 0, 1), (0, 1, 0), (1, 0, 0)),
             ((-1, 0, 0), (0, 1, 0), (0, 0, 1)), ((1, 0, 0), (0, 0, 1), (0, 1, 0))]
    verts, tris = [], []
    t = np.linspace(-0.5, 0.5, n + 1)
    for nrm, u, w in faces:
        nrm, u, w = np.array(nrm, float), np.array(u, float), np.array(w, float)
        base = sum(len(v) for v in verts)
        su, sw = np.meshgrid(t, t, indexing="xy")
        p = 0.5 * nrm + su.reshape(-1, 1) * u + sw.reshape(-1, 1) * w
        v = np.zeros((p.shape[0], 8), np.float32)
        v[:, 0:3] = p
        v[:, 3:6] = nrm
        v[:, 6] = su.reshape(-1) + 0.5
        v[:, 7] = sw.reshape(-1) + 0.5
        verts.append(v)
        i = np.arange(n)
        a = (i[:, None] * (n + 1) + i[None, :]).reshape(-1) + base
        b, c, d = a + 1, a + n + 1, a + n + 2
        q = np.concatenate([np.stack([a, b, d], 1), np.stack([a, d, c], 1)])
        # wind so that cross(p1 - p0, p2 - p0) points along the face normal
        allv = np.concatenate(verts)
        p0, p1, p2 = allv[q[0, 0] - 0, :3], allv[q[0, 1], :3], allv[q[0, 2], :3]
        if np.dot(np.cross(p1 - p0, p2 - p0), nrm) < 0:
            q = q[:, [0, 2, 1]]
        tris.append(q)
    return Mesh(np.concatenate(verts), np.concatenate(tris).astype(np.uint32))


def city(seed: int = 1, boxes: int = 20000, extent: float = 2000.0, box_tessellation: int = 4,
         ground_cells: int = 400, width: int = 3840, height: int = 2160) -> SceneNode:
    """Seeded synthetic city: `boxes` buildings on a square grid of lots over
    extent x extent metres, footprints U[6, 12] m with random yaw, heights
    log-normal (mu 2, sigma 0.7) m, albedo U[0.2, 0.8] grey-tinted; one
    tessellated box mesh (12 n^2 triangles) instanced for all of them, and a
    ground plane of 2 x ground_cells^2 triangles."""
    rng = np.random.default_rng(seed)
    s = SceneNode(name=f"city_{boxes}_seed{seed}")
    cell = extent / ground_cells
    ground = s.add_mesh(grid_mesh(np.zeros((ground_cells + 1, ground_cells + 1)), cell))
    s.add_instance(ground, s.add_material(Material((0.35, 0.35, 0.33))), s.add_transform(np.eye(4, dtype=np.float32)))
    box = s.add_mesh(tessellated_box(box_tessellation))
    lots = int(math.ceil(math.sqrt(boxes)))
    spacing = extent / lots
    palette = [s.add_material(Material(tuple(float(x) for x in rng.uniform(0.2, 0.8) * rng.uniform(0.9, 1.1, 3))))
               for _ in range(64)]
    k = 0
    for iz in range(lots):
        for ix in range(lots):
            if k >= boxes:
                break
            fx, fz = rng.uniform(6.0, 12.0, 2)
            hgt = float(np.exp(rng.normal(2.0, 0.7)))
            x = -0.5 * extent + (ix + 0.5) * spacing + rng.uniform(-0.15, 0.15) * spacing
            z = -0.5 * extent + (iz + 0.5) * spacing + rng.uniform(-0.15, 0.15) * spacing
            yaw = rng.uniform(0.0, 2.0 * math.pi)
            s.add_instance(box, palette[int(rng.integers(0, len(palette)))],
                           s.add_transform(make_transform((x, 0.5 * hgt, z), (0.0, yaw, 0.0), (fx, hgt, fz))))
            k += 1
    s.camera = _camera((0.0, 180.0, 0.55 * extent), (0.0, 0.0, 0.1 * extent), 55.0, width, height)
    s.lighting = Lighting.sun_elevation(30.0, azimuth_deg=40.0, irradiance=3.0, sky=0.5)
    return s


def batch_scenes(count: int = 64, seed: int = 1, tri_min: float = 1e3, tri_max: float = 5e5,
                 sites_min: int = 512, sites_max: int = 20480) -> list[tuple[SceneNode, int]]:
    """(scene, site count) pairs. Each scene is a terrain_boxes scene of about
    T triangles, T log-uniform in [tri_min, tri_max]: 95 % terrain grid and
    5 % boxes (12 triangles each)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        t = math.exp(rng.uniform(math.log(tri_min), math.log(tri_max)))
        boxes = max(1, int(0.05 * t / 12.0))
        grid = max(3, int(round(math.sqrt(0.95 * t / 2.0))) + 1)
        node = terrain_boxes(seed=seed * 1000 + i, grid=grid, boxes=boxes)
        out.append((node, int(rng.integers(sites_min, sites_max + 1))))
    return out


def surface_sites(scene_node: SceneNode, count: int, seed: int = 1, radius: float = 0.25,
                  double_sided_backs: bool = True):
    """Area-weighted random surface sites as probe records.

    Returns (probes SURFACE_PROBE_DTYPE[N], instances SURFACE_PROBE_INSTANCE_DTYPE[I]).
    Each site stores (primitive, bary.y, bary.z, instance << 8 | back flag);
    double-sided materials get a back record with the negated normal, as the
    reference's _make_probe_records does (surface_probes.py:1302-1345). The
    reference places sites by weighted sample elimination; this stand-in only
    needs valid sites on the surfaces.
    """
    rng = np.random.default_rng(seed)
    inst_area = []
    tri_world = []
    for mesh_id, _, transform_id in scene_node.instances:
        mesh = scene_node.meshes[mesh_id]
        m = scene_node.transforms[transform_id].astype(np.float64)
        p = mesh.vertices[:, 0:3].astype(np.float64) @ m[:3, :3].T + m[:3, 3]
        tri = p[mesh.indices.astype(np.int64)]
        area = 0.5 * np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1)
        tri_world.append((tri, area))
        inst_area.append(area.sum())
    inst_area = np.asarray(inst_area)
    inst_pick = rng.choice(len(inst_area), size=count, p=inst_area / inst_area.sum())
    records = []
    for inst in range(len(inst_area)):
        k = int((inst_pick == inst).sum())
        if k == 0:
            continue
        tri, area = tri_world[inst]
        prims = rng.choice(len(area), size=k, p=area / area.sum())
        u = rng.random((k, 2))
        su = np.sqrt(u[:, 0])
        b1 = (1.0 - u[:, 1]) * su
        b2 = u[:, 1] * su
        b0 = 1.0 - b1 - b2
        pos = b0[:, None] * tri[prims, 0] + b1[:, None] * tri[prims, 1] + b2[:, None] * tri[prims, 2]
        n = np.cross(tri[prims, 1] - tri[prims, 0], tri[prims, 2] - tri[prims, 0])
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        material = scene_node.materials[scene_node.instances[inst][1]]
        sides = 2 if (material.double_sided and double_sided_backs) else 1
        for side in range(sides):
            r = np.zeros(k, dtype=SURFACE_PROBE_DTYPE)
            sign = -1.0 if side == 1 else 1.0
            r["position_radius"][:, :3] = pos
            r["position_radius"][:, 3] = radius
            r["normal_side"][:, :3] = n * sign
            r["normal_side"][:, 3] = 1.0
            r["meta"][:, 0] = prims
            r["meta"][:, 1] = b1.astype(np.float32).view(np.uint32)
            r["meta"][:, 2] = b2.astype(np.float32).view(np.uint32)
            r["meta"][:, 3] = (SURFACE_PROBE_FLAG_BACK_SIDE if side else 0) | (inst << SURFACE_PROBE_INSTANCE_SHIFT)
            records.append(r)
    probes = np.concatenate(records)
    instances = np.zeros(len(scene_node.instances), dtype=SURFACE_PROBE_INSTANCE_DTYPE)
    instances["params"][:, 0] = radius
    return probes, instances
