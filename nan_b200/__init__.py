"""nan_b200: B200-native path integration for the Nan renderer's hot path.

Hand-written sm_100a CUDA kernels (libnan_b200.so, C ABI in
include/nan_b200.h) behind Python classes that keep the reference's pass API:

    PathTracer(device, scene).execute(stream, output, frame)
    TextureSpacePathTracer(device, scene, layout, samples_per_texel=1, max_bounces=3)
        .execute(stream, output, iteration, reset=False)
    SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=1, max_bounces=3)
        .execute(stream, field, attachments, iteration, reset=False)
    Accumulator(device).execute(stream, render_data, input, output, reset=False)
    MeshColorsRGB9E5Packer(device).execute(stream, source, destination, texel_count)

PyTorch tensors serve as device buffers; ``command_encoder`` is a CUDA stream.
"""

from .accumulator import Accumulator
from .cached_path_tracer import CachedPathTracer
from .camera import Camera, HaltonSamplePattern, halton
from .mesh_colors import (MESH_COLORS_INVALID_OFFSET, MESH_COLORS_PAYLOAD_SIZE, MESH_COLORS_SIDE_FLAG_DOUBLE_SIDED,
                          MeshColorsLayout, address_to_ij, barycentric_at, colors_per_patch, ij_to_address)
from .mesh_colors_resolve import MeshColorsResolve
from .mesh_colors_surface_filter import MeshColorsSurfaceFilter
from .mesh_colors_rgb9e5 import MeshColorsRGB9E5Packer
from .path_tracer import PathTracer
from .probe_batch import ProbeBatch
from .radiance_cache import RadianceCache
from .render_data import RenderData
from .scene import Device, Lighting, Scene
from .scene_node import Material, Mesh, SceneNode, make_transform
from .surface_probe_fields import (DIFFUSE_IRRADIANCE_ATTACHMENTS, DIFFUSE_IRRADIANCE_RGB_FIELD,
                                   SurfaceProbeAttachments, SurfaceProbeFieldBuffers, SurfaceProbeRuntimeBuffers)
from .surface_probe_prt import (SurfaceProbePrtBaker, SurfaceProbePrtEvaluator, evaluate_prt_l2_rgb,
                               surface_probe_sh_l2_basis)
from .surface_probe_path_tracer import SurfaceProbeDiffuseIrradianceBaker, SurfaceProbePathTracer
from .surface_probe_layout import SurfaceProbeLayout, SurfaceProbeSiteLayout
from .surface_probe_resolve import SurfaceProbeResolve
from .surface_probe_resources import SurfaceProbeGpuGeometry
from .texture_space_path_tracer import TextureSpacePathTracer
from .visibility import PMRVisibilitySHSampler, trace_pmr_visibility_sh, visibility_ray_table

__all__ = [
    "Accumulator", "CachedPathTracer", "Camera", "Device", "HaltonSamplePattern", "Lighting", "Material", "Mesh", "MeshColorsLayout",
    "MeshColorsRGB9E5Packer", "MeshColorsResolve", "MeshColorsSurfaceFilter", "PathTracer", "ProbeBatch", "RadianceCache", "RenderData", "Scene", "SceneNode", "SurfaceProbeAttachments",
    "SurfaceProbeDiffuseIrradianceBaker", "SurfaceProbeFieldBuffers", "SurfaceProbeGpuGeometry",
    "SurfaceProbePathTracer", "SurfaceProbePrtBaker", "SurfaceProbeResolve", "SurfaceProbeLayout", "SurfaceProbeSiteLayout", "SurfaceProbePrtEvaluator", "evaluate_prt_l2_rgb", "surface_probe_sh_l2_basis", "SurfaceProbeRuntimeBuffers", "TextureSpacePathTracer", "PMRVisibilitySHSampler", "trace_pmr_visibility_sh", "visibility_ray_table", "address_to_ij",
    "barycentric_at", "colors_per_patch", "halton", "ij_to_address", "make_transform",
    "DIFFUSE_IRRADIANCE_ATTACHMENTS", "DIFFUSE_IRRADIANCE_RGB_FIELD", "MESH_COLORS_INVALID_OFFSET",
    "MESH_COLORS_PAYLOAD_SIZE", "MESH_COLORS_SIDE_FLAG_DOUBLE_SIDED",
]
