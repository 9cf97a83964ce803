"""Timing of the passes that consume the accumulated caches, on the
texel-tracer workload's scene and slots: Mesh Colors resolve (16-byte slots
and RGB9E5), the RGB9E5 pack, one surface-filter pass over every slot, and
on a probe layout of the same scene built as the reference builds it
(adaptive weighted sample elimination of 5x oversampled candidates for
20,480 sites, deficit repair, protected closure): the irradiance and PRT L2
bakers (16 spp, 3 bounces), the PRT evaluation and the probe resolve. Every
pass runs once untimed, then `frames` times between CUDA events on the
launching stream; rates are per second of that device time.
"""

from __future__ import annotations

import math
import time


def measure(device, scene, node, layout, slots, *, frames: int = 5, width: int = 1920, height: int = 1080,
            probe_sites: int = 20480) -> dict:
    import torch

    from nan_b200.mesh_colors_resolve import MeshColorsResolve
    from nan_b200.mesh_colors_rgb9e5 import MeshColorsRGB9E5Packer
    from nan_b200.mesh_colors_surface_filter import MeshColorsSurfaceFilter
    from nan_b200.render_data import RenderData
    from nan_b200.surface_probe_fields import (DIFFUSE_PRT_ATTACHMENTS, DIFFUSE_PRT_L2_RGB_FIELD,
                                       SurfaceProbeRuntimeBuffers)
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout
    from nan_b200.surface_probe_path_tracer import SurfaceProbeDiffuseIrradianceBaker
    from nan_b200.surface_probe_prt import SurfaceProbePrtBaker, SurfaceProbePrtEvaluator
    from nan_b200.surface_probe_resolve import SurfaceProbeResolve
    from nan_b200.surface_probe_resources import SurfaceProbeGpuGeometry
    from nan_b200.texture_space_path_tracer import TextureSpacePathTracer

    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn) -> float:
        fn(0)
        torch.cuda.synchronize()
        e0.record(stream)
        for f in range(1, frames + 1):
            fn(f)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / frames

    res: dict = {"frames": frames, "screen": f"{width}x{height}"}
    node.camera.begin_frame(width, height)
    out = torch.zeros((height, width, 4), dtype=torch.float32, device=device.torch_device)
    tracer = TextureSpacePathTracer(device, scene, layout)
    mcr = MeshColorsResolve(device, scene, layout, tracer)
    px = width * height
    ms = timed(lambda f: mcr.execute(stream, slots, out))
    res["mesh_colors_resolve"] = {"ms": ms, "mpixels_per_s": px / (ms * 1e3)}
    packed = torch.zeros(layout.total_payload_count, dtype=torch.int32, device=device.torch_device)
    packer = MeshColorsRGB9E5Packer(device)
    ms = timed(lambda f: packer.execute(stream, slots, packed, layout.total_payload_count))
    res["rgb9e5_pack"] = {"ms": ms, "slots": layout.total_payload_count,
                          "gb_per_s": layout.total_payload_count * 20 / (ms * 1e6)}
    ms = timed(lambda f: mcr.execute_frozen(stream, packed, out))
    res["mesh_colors_frozen_resolve"] = {"ms": ms, "mpixels_per_s": px / (ms * 1e3)}
    filt = MeshColorsSurfaceFilter(device, scene, layout)
    dst = torch.empty_like(slots)
    ms = timed(lambda f: filt.execute(stream, slots, dst))
    texels = layout.total_surface_texels
    res["surface_filter"] = {"ms": ms, "texels": texels, "gtexels_per_s": texels / (ms * 1e6),
                             "gb_per_s_at_32_bytes_per_texel": texels * 32 / (ms * 1e6)}
    del dst, packed

    t0 = time.perf_counter()
    placement: dict = {}
    sites = SurfaceProbeSiteLayout.build_wse(node, probe_sites, device=device, seed=1, profile=placement)
    res["probe_site_placement"] = dict(placement, total_s=time.perf_counter() - t0)
    geometry = SurfaceProbeGpuGeometry.create(device, sites)
    n = sites.total_probe_count
    rd = RenderData(device)
    rt = SurfaceProbeRuntimeBuffers.acquire(rd, n)
    baker = SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=16, max_bounces=3)
    ms = timed(lambda f: baker.execute(stream, rt.field, rt.attachments, f, reset=(f == 0)))
    res["probe_irradiance_bake"] = {"ms": ms, "probes": n, "samples_per_probe": 16,
                                    "msamples_per_s": n * 16 / (ms * 1e3)}
    prt = SurfaceProbeRuntimeBuffers.acquire(rd, n, field_desc=DIFFUSE_PRT_L2_RGB_FIELD,
                                             attachment_descs=DIFFUSE_PRT_ATTACHMENTS, resource_prefix="prt")
    prt_baker = SurfaceProbePrtBaker(device, scene, geometry, samples_per_probe=16, max_bounces=3)
    ms = timed(lambda f: prt_baker.execute(stream, prt.field, prt.attachments, f, reset=(f == 0)))
    res["prt_l2_bake"] = {"ms": ms, "probes": n, "samples_per_probe": 16, "msamples_per_s": n * 16 / (ms * 1e3)}
    evaluator = SurfaceProbePrtEvaluator(device, scene, geometry)
    ms = timed(lambda f: evaluator.execute(stream, rd, prt.field, prt.attachments))
    res["prt_evaluate"] = {"ms": ms, "probes": n}
    resolve = SurfaceProbeResolve(device, scene, sites, geometry)
    ms = timed(lambda f: resolve.execute(stream, rt.field, rt.attachments, out))
    res["probe_resolve"] = {"ms": ms, "mpixels_per_s": px / (ms * 1e3), "probes": n,
                            "kernel_radius_m": float(sites.instance_infos[0].kernel_radius),
                            "sites_per_kernel_disc": math.pi * 2.5 ** 2}
    device.check()
    return res


def main(argv=None) -> None:
    """Standalone run on the texel-tracer workload (seeded terrain, grid 313,
    500 boxes; 16 texels per unit), slots filled by 4 texel iterations; prints
    one JSON line."""
    import argparse
    import json

    import torch

    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout
    from nan_b200.scene import Device, Scene
    from nan_b200.texture_space_path_tracer import TextureSpacePathTracer

    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=5)
    ap.add_argument("--grid", type=int, default=313)
    ap.add_argument("--boxes", type=int, default=500)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    args = ap.parse_args(argv)
    device = Device(0)
    node = scenes.terrain_boxes(seed=1, grid=args.grid, boxes=args.boxes)
    scene = Scene(device, node)
    layout = MeshColorsLayout.build(node, texels_per_unit=16.0, min_resolution=4, max_resolution=64)
    slots = torch.zeros((layout.total_payload_count, 4), dtype=torch.int32, device=device.torch_device)
    tracer = TextureSpacePathTracer(device, scene, layout, samples_per_texel=1, max_bounces=3)
    for it in range(4):
        tracer.execute(None, slots, it, reset=(it == 0))
    print(json.dumps(measure(device, scene, node, layout, slots, frames=args.frames, width=args.width,
                             height=args.height)))


if __name__ == "__main__":
    main()
