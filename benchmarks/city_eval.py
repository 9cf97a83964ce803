"""One frame of the large workload on the seeded 4.16 M-triangle city
(scenes.city): the screen at 3840x2160 with 4 spp and 5 path vertices (the
learned-cache path tracer, and the plain one for comparison), a 20,480-site
surface-probe pass (sites by the adaptive weighted sample elimination of 5x
oversampled candidates on the GPU, no repair sites; 64 spp, 3 bounces, compensated sums, batched launch
with one RNG stream per sample, one wavefront path per probe and sample) and
a Mesh Colors texel pass over the whole city (about 12.6 M texels, 1 sample,
3 bounces). Every pass is timed with CUDA events on the launching stream
after one warm-up frame; rays are counted on the device.
"""

from __future__ import annotations

import time


def measure(device, frames: int = 2, width: int = 3840, height: int = 2160, spp: int = 4) -> dict:
    import torch

    from nan_b200 import scenes as sc
    from nan_b200.accumulator import Accumulator
    from nan_b200.cached_path_tracer import CachedPathTracer
    from nan_b200.radiance_cache import scene_bounds
    from nan_b200.mesh_colors import MeshColorsLayout
    from nan_b200.path_tracer import PathTracer
    from nan_b200.probe_batch import ProbeBatch
    from nan_b200.radiance_cache import RadianceCache
    from nan_b200.render_data import RenderData
    from nan_b200.scene import Scene
    from nan_b200.surface_probe_fields import SurfaceProbeRuntimeBuffers
    from nan_b200.surface_probe_path_tracer import SurfaceProbeDiffuseIrradianceBaker
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout
    from nan_b200.surface_probe_resources import SurfaceProbeGpuGeometry
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler
    from nan_b200.texture_space_path_tracer import TextureSpacePathTracer

    t0 = time.perf_counter()
    node = sc.city(width=width, height=height)
    node.lighting.ray_t_max = 5000.0  # the city's diagonal exceeds the reference's 1000
    scene = Scene(device, node)
    layout = MeshColorsLayout.build(node, texels_per_unit=0.1, min_resolution=1, max_resolution=64)
    host_s = time.perf_counter() - t0
    t1 = time.perf_counter()
    placement: dict = {}
    # the config's 20,480 sites: the adaptive elimination's output, without
    # repair or closure sites
    sites = SurfaceProbeSiteLayout.build_wse(node, 20480, sampler=SurfaceProbeSampler(device), seed=1,
                                             repair_min_gather=0, profile=placement)
    placement["total_s"] = time.perf_counter() - t1
    info = scene.info()
    rd = RenderData(device)
    dev = device.torch_device
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, ctx):
        fn(0)
        torch.cuda.synchronize()
        ctx.read_counters(reset=True)
        e0.record(stream)
        for f in range(1, frames + 1):
            fn(f)
        e1.record(stream)
        e1.synchronize()
        c = ctx.read_counters(reset=True)
        ms = e0.elapsed_time(e1) / frames
        rays = (c["extend_rays"] + c["shadow_rays"]) / frames
        return {"ms": ms, "rays": rays, "mrays_per_s": rays / (ms * 1e3)}

    out = torch.zeros((height, width, 4), dtype=torch.float32, device=dev)
    disp = torch.zeros_like(out)
    acc = Accumulator(device)
    plain = PathTracer(device, scene, max_vertices=5)

    def screen_plain(f):
        for k in range(spp):
            node.camera.begin_frame(width, height)
            plain.execute(stream, out, spp * f + k)
            acc.execute(stream, rd, out, disp, reset=(k == 0))

    lo, hi = scene_bounds(scene)
    cache = RadianceCache(device, lo, hi)
    cached = CachedPathTracer(device, scene, cache, cache_vertex=1, max_vertices=5, train_samples=65536,
                              train_batch=16384)

    def screen_cached(f):
        for k in range(spp):
            node.camera.begin_frame(width, height)
            cached.execute(stream, out, spp * f + k)
            acc.execute(stream, rd, out, disp, reset=(k == 0))

    res = {"screen_plain": timed(screen_plain, scene.context)}
    res["screen_learned_cache"] = timed(screen_cached, scene.context)

    geometry = SurfaceProbeGpuGeometry.create(device, sites)
    baker = SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=64, max_bounces=3,
                                               compensated=True)
    rt = SurfaceProbeRuntimeBuffers.acquire(rd, geometry.probe_count)
    batch = ProbeBatch(device, [(baker, rt.field, rt.attachments)], independent_samples=True, wavefront=True)
    tuned = batch.autotune(64, 3)
    res["probes"] = timed(lambda f: batch.execute(stream, f, 64, 3, reset=(f == 0)), batch.context)
    res["probes"]["autotune"] = tuned

    slots = torch.zeros((layout.total_payload_count, 4), dtype=torch.int32, device=dev)
    texels = TextureSpacePathTracer(device, scene, layout, samples_per_texel=1, max_bounces=3)
    res["texels"] = timed(lambda f: texels.execute(stream, slots, f, reset=(f == 0)), scene.context)
    device.check()
    frame_ms = res["screen_learned_cache"]["ms"] + res["probes"]["ms"] + res["texels"]["ms"]
    return {
        "scene": f"seeded city: 20,000 boxes (log-normal heights mu 2, sigma 0.7) on a 2 km grid + ground, "
                 f"{info['triangle_count']} triangles, sun 30 deg + sky 0.5, t_max 5000",
        "bvh_build_ms": info["build_ms"], "host_setup_s": host_s, "site_placement": placement,
        "screen": f"{width}x{height}, {spp} spp, 5 path vertices", "probe_sites": int(geometry.probe_count),
        "texels": int(layout.total_surface_texels), "passes": res,
        "frame_ms_learned_screen_probes_texels": frame_ms,
    }
