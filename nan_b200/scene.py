"""Device, lighting and the GPU scene (the reference's Scene, scene.py:32-1382).

``Scene(device, scene_node)`` uploads the scene in the reference's record
layouts as torch tensors (buffers only) and builds the BVH on the GPU through
``nan_scene_build``. The tensors stay alive as long as the Scene, because the
shading code reads them in place.
"""

from __future__ import annotations

import ctypes
import math
import weakref
from dataclasses import dataclass, field

import numpy as np

from . import _native
from ._native import NanLighting, NanSceneDesc, NanSceneInfo, check, lib, ptr, stream_handle
from .scene_node import SceneNode


class Device:
    """One CUDA device plus the native context used by every pass on it."""

    def __init__(self, index: int = 0):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("nan_b200 needs a CUDA device (there is no CPU path)")
        self.index = int(index)
        self.torch_device = torch.device("cuda", self.index)
        self.context = _native.Context(self.index)
        self._contexts = weakref.WeakSet()

    def new_context(self) -> _native.Context:
        """A further native context on this device (one per scene/BVH)."""
        ctx = _native.Context(self.index)
        self._contexts.add(ctx)
        return ctx

    def synchronize(self) -> None:
        import torch

        torch.cuda.synchronize(self.torch_device)

    def check(self, stream=None) -> None:
        """Raise if a kernel on this device reported a device-side limit or a
        bad record since the last check (every context of the device)."""
        self.context.check(stream)
        for ctx in list(self._contexts):
            ctx.check(stream)

    @property
    def launch_count(self) -> int:
        return self.context.launch_count + sum(c.launch_count for c in list(self._contexts))


# The reference atmosphere (atmosphere.slang:4-8): radii in megametres, the
# view 200 m above the ground.
GROUND_RADIUS_MM = 6.360
ATMOSPHERE_RADIUS_MM = 6.460
VIEW_HEIGHT_MM = GROUND_RADIUS_MM + 0.0002


def sky_view_horizon_angle(view_height: float = VIEW_HEIGHT_MM, ground_radius: float = GROUND_RADIUS_MM) -> float:
    """acos(sqrt(h^2 - R^2) / h) - pi/2 in float32 (scene.slang:474)."""
    f = np.float32
    h, r = f(view_height), f(ground_radius)
    c = np.sqrt(h * h - r * r) / h
    return float(f(np.arccos(np.clip(c, f(-1), f(1)))) - f(0.5) * f(math.pi))


def sun_transmittance_from_lut(lut, sun_direction, up=(0.0, 1.0, 0.0), view_height: float = VIEW_HEIGHT_MM,
                               ground_radius: float = GROUND_RADIUS_MM,
                               atmosphere_radius: float = ATMOSPHERE_RADIUS_MM) -> tuple:
    """get_sun_transmittance_at_view (scene.slang:997-1009): the
    transmittance LUT (float32 [H, W, >=3], e.g. 64 x 256) read bilinearly
    with clamp-to-edge at u = 0.5 + 0.5 cos(sun zenith), v = the view
    height's fraction of the atmosphere. Returns the rgb factor for
    Lighting.sun_transmittance."""
    t = np.asarray(lut.cpu() if hasattr(lut, "cpu") else lut, dtype=np.float32)
    d = np.asarray(sun_direction, np.float64)
    mu = float(np.dot(d / np.linalg.norm(d), np.asarray(up, np.float64)))
    u = min(max(0.5 + 0.5 * mu, 0.0), 1.0)
    v = min(max((view_height - ground_radius) / (atmosphere_radius - ground_radius), 0.0), 1.0)
    h, w = t.shape[0], t.shape[1]
    x, y = u * w - 0.5, v * h - 0.5
    x0, y0 = math.floor(x), math.floor(y)
    fx, fy = x - x0, y - y0

    def at(i, j):
        return t[min(max(j, 0), h - 1), min(max(i, 0), w - 1), :3].astype(np.float64)

    top = at(x0, y0) * (1 - fx) + at(x0 + 1, y0) * fx
    bottom = at(x0, y0 + 1) * (1 - fx) + at(x0 + 1, y0 + 1) * fx
    return tuple(float(c) for c in top * (1 - fy) + bottom * fy)


@dataclass
class Lighting:
    """Directional sun and sky.

    Defaults follow Scene.__init__ (scene.py:135-147): sun toward
    (0, 0.5, 0.866), color white, intensity pi, half apex angle 0.26785 deg.
    The sky is the constant `sky_radiance`, or, with `sky_view_lut` set (a
    float32 [H, W, 4] CUDA tensor, the reference's sky-view LUT), the LUT
    looked up per miss direction as sample_sky_lut does (scene.slang:469-518).
    The sun transmittance is one value per frame in the reference
    (get_sun_transmittance_at_view reads its LUT at the fixed view position,
    scene.slang:997-1009): `sun_transmittance_from_lut` computes it.
    """

    sun_direction: tuple = (0.0, 0.5, 0.866)
    sun_cos_half_angle: float = math.cos(math.radians(0.5357 / 2.0))
    sun_color: tuple = (1.0, 1.0, 1.0)
    sun_intensity: float = math.pi
    sun_transmittance: tuple = (1.0, 1.0, 1.0)
    ray_t_max: float = 1000.0
    sky_radiance: tuple = (0.0, 0.0, 0.0)
    sun_disk: bool = True
    # screen tracer only, not in the reference: NEE toward the scene's emissive
    # triangles with MIS (Scene.enable_area_lights builds the table)
    area_nee: bool = False
    sky_view_lut: object = None
    sky_view_up: tuple = (0.0, 1.0, 0.0)
    sky_view_horizon_angle: float | None = None  # None: the reference atmosphere's view height

    def __post_init__(self):
        d = np.asarray(self.sun_direction, dtype=np.float64)
        n = np.linalg.norm(d)
        self.sun_direction = tuple(float(x) for x in (d / n if n > 0 else d))

    @property
    def flags(self) -> int:
        return (1 if self.sun_disk else 0) | (2 if self.area_nee else 0)

    def to_struct(self) -> NanLighting:
        s = NanLighting()
        s.sun_direction[:] = [float(x) for x in self.sun_direction]
        s.sun_cos_half_angle = float(self.sun_cos_half_angle)
        s.sun_color[:] = [float(x) for x in self.sun_color]
        s.sun_intensity = float(self.sun_intensity)
        s.sun_transmittance[:] = [float(x) for x in self.sun_transmittance]
        s.ray_t_max = float(self.ray_t_max)
        s.sky_radiance[:] = [float(x) for x in self.sky_radiance]
        s.flags = self.flags
        lut = self.sky_view_lut
        if lut is not None:
            import torch

            if not (isinstance(lut, torch.Tensor) and lut.is_cuda and lut.dtype == torch.float32 and lut.dim() == 3
                    and lut.shape[2] == 4 and lut.is_contiguous()):
                raise ValueError("sky_view_lut must be a contiguous float32 [H, W, 4] CUDA tensor")
            s.sky_view_lut = int(lut.data_ptr())
            s.sky_view_height, s.sky_view_width = int(lut.shape[0]), int(lut.shape[1])
        s.sky_view_up[:] = [float(x) for x in self.sky_view_up]
        s.sky_view_horizon_angle = (sky_view_horizon_angle() if self.sky_view_horizon_angle is None
                                    else float(self.sky_view_horizon_angle))
        return s

    @classmethod
    def sun_elevation(cls, elevation_deg: float, azimuth_deg: float = 0.0, irradiance: float = 3.0,
                      sky: float = 0.5, **kw) -> "Lighting":
        """Sun at the given elevation with color*intensity = irradiance."""
        e, a = math.radians(elevation_deg), math.radians(azimuth_deg)
        direction = (math.cos(e) * math.sin(a), math.sin(e), math.cos(e) * math.cos(a))
        return cls(sun_direction=direction, sun_intensity=irradiance, sky_radiance=(sky, sky, sky), **kw)


class Scene:
    """Scene buffers on the GPU + BVH (replaces Scene.__init__/bind)."""

    def __init__(self, device: Device, scene_node: SceneNode, lighting: Lighting | None = None, stream=None,
                 bvh_builder: str = "sah"):
        import torch

        self.device = device
        self.scene_node = scene_node
        self.camera = scene_node.camera
        self.lighting = lighting or scene_node.lighting or Lighting()
        self.frame_index = 0
        self.bvh_builder = bvh_builder
        packed = scene_node.pack()
        self.host = packed
        td = device.torch_device
        self.vertices = torch.from_numpy(packed["vertices"]).to(td)
        self.indices = torch.from_numpy(packed["indices"].view(np.int32)).to(td)
        self.mesh_descs = torch.from_numpy(packed["mesh_descs"].view(np.int32)).to(td)
        self.instance_descs = torch.from_numpy(packed["instance_descs"].view(np.int32)).to(td)
        self.transforms = torch.from_numpy(packed["transforms"]).to(td)
        self.inverse_transposes = torch.from_numpy(packed["inverse_transposes"]).to(td)
        self.materials = torch.from_numpy(packed["materials"]).to(td)
        desc = NanSceneDesc()
        desc.vertices = ptr(self.vertices)
        desc.vertex_count = packed["vertices"].shape[0]
        desc.indices = ptr(self.indices)
        desc.index_triangle_count = packed["indices"].shape[0]
        desc.mesh_descs = ptr(self.mesh_descs)
        desc.mesh_count = packed["mesh_descs"].shape[0]
        desc.instance_descs = ptr(self.instance_descs)
        desc.instance_count = packed["instance_descs"].shape[0]
        desc.transforms = ptr(self.transforms)
        desc.inverse_transposes = ptr(self.inverse_transposes)
        desc.transform_count = packed["transforms"].shape[0]
        desc.materials = ptr(self.materials)
        desc.material_count = packed["materials"].shape[0]
        self._desc = desc
        self._context = device.new_context()
        self._context.configure(bvh_builder=bvh_builder)
        check(lib().nan_scene_build(self._context.handle, ctypes.byref(desc), stream_handle(stream)))

    @property
    def context(self) -> _native.Context:
        """The native context that owns this scene's BVH."""
        return self._context

    def configure(self, integrator: str = "wavefront", trace_blocks_per_sm: int = 0,
                  max_paths_in_flight: int = 0, bvh_width: int = 2, kernel_timing: bool = False,
                  ray_order: int = 0, traversal: int = 0) -> None:
        """Integrator form for passes on this scene: "wavefront" (default) or
        "megakernel" (one thread per pixel/texel/probe), launch shapes, the
        traversed node width (2: binary, the default; 8: compressed wide nodes),
        per-stage CUDA-event timing (read with context.read_kernel_times) and
        the wavefront's ray order (1: extend queue regrouped by direction
        octant)."""
        self._context.configure(integrator, trace_blocks_per_sm, max_paths_in_flight, self.bvh_builder, bvh_width,
                                kernel_timing, ray_order, traversal)

    def area_light_table(self):
        """(f32[L, 16], power): every emissive triangle of the scene in world
        space -- v0, inclusive cdf; v1 - v0, area; v2 - v0, luminance;
        emission -- with selection weights area * luminance."""
        node = self.scene_node
        rows = []
        for mesh_id, mat_id, transform_id in node.instances:
            mat = node.materials[mat_id]
            e = np.asarray(mat.emissive, dtype=np.float32)
            lum = (np.float32(0.2126) * e[0] + np.float32(0.7152) * e[1]) + np.float32(0.0722) * e[2]
            if not lum > 0:
                continue
            mesh = node.meshes[mesh_id]
            m = node.transforms[transform_id].astype(np.float32)
            p = (mesh.vertices[:, 0:3].astype(np.float32) @ m[:3, :3].T + m[:3, 3]).astype(np.float32)
            tri = p[mesh.indices.astype(np.int64)]
            e1 = (tri[:, 1] - tri[:, 0]).astype(np.float32)
            e2 = (tri[:, 2] - tri[:, 0]).astype(np.float32)
            area = (0.5 * np.linalg.norm(np.cross(e1.astype(np.float64), e2.astype(np.float64)), axis=1))
            r = np.zeros((tri.shape[0], 16), np.float32)
            r[:, 0:3], r[:, 4:7], r[:, 8:11] = tri[:, 0], e1, e2
            r[:, 7] = area
            r[:, 11] = lum
            r[:, 12:15] = e
            rows.append(r)
        if not rows:
            return np.zeros((0, 16), np.float32), 0.0
        t = np.concatenate(rows)
        w = t[:, 7].astype(np.float64) * t[:, 11].astype(np.float64)
        power = float(np.float32(w.sum()))
        cdf = np.cumsum(w) / w.sum()
        cdf[-1] = 1.0
        t[:, 3] = cdf.astype(np.float32)
        return t, power

    def enable_area_lights(self, enabled: bool = True) -> None:
        """Screen tracer: NEE toward the emissive triangles with MIS (an option
        beyond the reference, whose path tracer reaches emitters by BSDF
        sampling only). Sets lighting.area_nee."""
        import torch

        if enabled:
            table, power = self.area_light_table()
            self._area_lights = torch.from_numpy(table).to(self.device.torch_device)
            self._area_power = power
            check(lib().nan_ctx_set_area_lights(self.context.handle, ptr(self._area_lights), table.shape[0],
                                                ctypes.c_float(power)))
        else:
            check(lib().nan_ctx_set_area_lights(self.context.handle, None, 0, ctypes.c_float(0.0)))
        self.lighting.area_nee = bool(enabled)

    def trace_points(self, points, iteration: int, samples: int = 1, max_bounces: int = 3, out=None, stream=None,
                     indirect_only: bool = False):
        """Irradiance at surface points f32[N, 4] (b1, b2, instance bits,
        primitive bits | back << 31): f32[N, 4] (E rgb, 0; w = -1 where the
        instance is ~0). The estimator of TextureSpacePathTracer at given points."""
        import torch

        n = int(points.shape[0])
        if out is None:
            out = torch.empty((n, 4), dtype=torch.float32, device=points.device)
        self.context.reserve_paths(max(n, 1))
        light = self.lighting.to_struct()
        check(lib().nan_trace_points(self.context.handle, ptr(points), n, ptr(out), int(iteration) & 0xFFFFFFFF,
                                     int(samples), int(max_bounces), int(bool(indirect_only)), ctypes.byref(light),
                                     stream_handle(stream)))
        return out

    def info(self) -> dict:
        info = NanSceneInfo()
        check(lib().nan_scene_info(self.context.handle, ctypes.byref(info)))
        return {name: getattr(info, name) for name, _ in NanSceneInfo._fields_}

    @property
    def triangle_count(self) -> int:
        return int(self.info()["triangle_count"])

    def update(self) -> None:
        """Per-frame update (scene.py:1213-1216)."""
        self.frame_index += 1

    def world_triangles(self):
        import torch

        n = self.triangle_count
        out = torch.empty((n, 9), dtype=torch.float32, device=self.device.torch_device)
        check(lib().nan_scene_world_triangles(self.context.handle, ptr(out), stream_handle(None)))
        return out

    def intersect(self, rays, stream=None):
        """Closest hit of rays f32[N,8] -> (ids i32[N,4], tb f32[N,3])."""
        import torch

        rays = rays.contiguous()
        n = rays.shape[0]
        ids = torch.empty((n, 4), dtype=torch.int32, device=rays.device)
        tb = torch.empty((n, 3), dtype=torch.float32, device=rays.device)
        check(lib().nan_intersect(self.context.handle, ptr(rays), n, ptr(ids), ptr(tb), stream_handle(stream)))
        return ids, tb

    def occluded(self, rays, stream=None):
        """Visibility (1 = unoccluded) of rays f32[N,8]."""
        import torch

        rays = rays.contiguous()
        n = rays.shape[0]
        vis = torch.empty((n,), dtype=torch.float32, device=rays.device)
        check(lib().nan_occluded(self.context.handle, ptr(rays), n, ptr(vis), stream_handle(stream)))
        return vis
