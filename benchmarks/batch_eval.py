"""Multi-scene surface-probe baking: one batched persistent launch (direct
and replayed from a CUDA graph) against one baker dispatch per scene.

Every frame bakes every site of every scene (samples_per_probe cosine
samples, max_bounces bounces, compensated running means). The batched
launch runs in both sample modes: one RNG stream per probe (the reference's,
bit-exact with the per-scene baker) and one stream per sample (a warp per
probe). Frames are timed
with CUDA events on the launching stream after one warm-up frame; rays are
counted on the device.
"""

from __future__ import annotations

import concurrent.futures
import os
import threading
import time


def _sites_layout(probes, pinst):
    import numpy as np

    layout = type("SiteLayout", (), {})()
    layout.probes, layout.instance_gpu_data = probes, pinst
    layout.nodes = np.zeros((1, 4), np.uint32)
    layout.triangle_vertex_probes = np.zeros((1, 4), np.uint32)
    layout.total_probe_count = probes.shape[0]
    layout.instance_infos = list(range(pinst.shape[0]))
    return layout


def measure(device, count: int = 64, seed: int = 1, samples_per_probe: int = 64, max_bounces: int = 3,
            frames: int = 3, tri_max: float = 5e5) -> dict:
    import torch

    from nan_b200 import scenes as sc
    from nan_b200.probe_batch import ProbeBatch
    from nan_b200.render_data import RenderData
    from nan_b200.scene import Scene
    from nan_b200.surface_probe_fields import SurfaceProbeRuntimeBuffers
    from nan_b200.surface_probe_path_tracer import SurfaceProbeDiffuseIrradianceBaker
    from nan_b200.surface_probe_resources import SurfaceProbeGpuGeometry

    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    # the synthetic scenes are the input: generated before the set-up clock
    t0 = time.perf_counter()
    scene_nodes = list(sc.batch_scenes(count, seed, tri_max=tri_max))
    generation_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    placement = {"candidates": 0, "base_sites": 0, "repair_sites": 0, "protected_sites": 0, "density_prepass_s": 0.0,
                 "candidates_s": 0.0, "elimination_s": 0.0, "repair_s": 0.0, "support_s": 0.0, "packing_s": 0.0}
    # The scenes are independent and each placement is seeded per scene, so
    # they are set up by a few worker threads (one sampler context each): the
    # host's numpy work and the library's GPU calls release the GIL and
    # overlap. The results do not depend on the number of workers.
    workers = max(1, min(8, (os.cpu_count() or 1) // 2))
    local = threading.local()

    def set_up(i):
        node, n_sites = scene_nodes[i]
        if not hasattr(local, "sampler"):
            local.sampler = SurfaceProbeSampler(device)
        scene = Scene(device, node)
        prof: dict = {}
        # the config's sites: the adaptive elimination's output at the scene's
        # target, without repair or closure sites
        layout = SurfaceProbeSiteLayout.build_wse(node, n_sites, sampler=local.sampler, seed=seed + i,
                                                  repair_min_gather=0, profile=prof)
        geometry = SurfaceProbeGpuGeometry.create(device, layout)
        baker = SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=samples_per_probe,
                                                   max_bounces=max_bounces, compensated=True)
        rt = SurfaceProbeRuntimeBuffers.acquire(RenderData(device), geometry.probe_count)
        return (scene, baker, rt.field, rt.attachments), prof, int(geometry.probe_count)

    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as pool:
        done = list(pool.map(set_up, range(len(scene_nodes))))
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    items = [d[0] for d in done]
    for _, prof, _ in done:
        for k in placement:
            placement[k] += prof.get(k, 0)
    tris = [item[0].triangle_count for item in items]
    sites = [d[2] for d in done]
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

    # one baker dispatch per scene (the reference's shape), wavefront integrator
    def per_scene(f):
        for scene, baker, field, att in items:
            baker.execute(stream, field, att, f, reset=(f == 0))

    for scene, *_ in items:
        scene.context.read_counters(reset=True)
    per_scene_ms = timed(per_scene)
    per_scene_rays = sum(sum(v for k, v in s.context.read_counters(reset=True).items()
                             if k in ("extend_rays", "shadow_rays")) for s, *_ in items) / (frames + 1)
    # the same, one thread per probe (the kernel the batch runs, one launch per scene)
    for scene, *_ in items:
        scene.configure("megakernel")
    per_scene_mk_ms = timed(per_scene)
    for scene, *_ in items:
        scene.configure("wavefront")
        scene.context.read_counters(reset=True)

    batch = ProbeBatch(device, [(b, f, a) for _, b, f, a in items])
    tuned = batch.autotune(samples_per_probe, max_bounces)
    batch.context.read_counters(reset=True)
    batch_ms = timed(lambda f: batch.execute(stream, f, samples_per_probe, max_bounces, reset=(f == 0)))
    c = batch.context.read_counters(reset=True)
    batch_rays = (c["extend_rays"] + c["shadow_rays"]) / (frames + 1)
    batch.capture(0, True, samples_per_probe, max_bounces)
    graph_ms = timed(lambda f: batch.replay(1, stream))
    batch.close()
    # the same sample sequence as one multi-scene wavefront
    wf = ProbeBatch(device, [(b, f, a) for _, b, f, a in items], wavefront=True)
    tuned_wf = wf.autotune(samples_per_probe, max_bounces)
    wf.capture(0, True, samples_per_probe, max_bounces)
    wf.context.read_counters(reset=True)
    wf_ms = timed(lambda f: wf.replay(1, stream))
    c = wf.context.read_counters(reset=True)
    wf_rays = (c["extend_rays"] + c["shadow_rays"]) / (frames + 1)
    wf.close()
    # independent samples on the wavefront: one path per (probe, sample)
    wfi = ProbeBatch(device, [(b, f, a) for _, b, f, a in items], independent_samples=True, wavefront=True)
    tuned_wfi = wfi.autotune(samples_per_probe, max_bounces)
    wfi.capture(0, True, samples_per_probe, max_bounces)
    wfi.context.read_counters(reset=True)
    wfi_ms = timed(lambda f: wfi.replay(1, stream))
    c = wfi.context.read_counters(reset=True)
    wfi_rays = (c["extend_rays"] + c["shadow_rays"]) / (frames + 1)
    wfi.close()
    # one RNG stream per sample: a warp traces 32 samples of one probe at once
    ind = ProbeBatch(device, [(b, f, a) for _, b, f, a in items], independent_samples=True)
    tuned_ind = ind.autotune(samples_per_probe, max_bounces)
    ind.capture(0, True, samples_per_probe, max_bounces)
    ind.context.read_counters(reset=True)
    ind_ms = timed(lambda f: ind.replay(1, stream))
    c = ind.context.read_counters(reset=True)
    ind_rays = (c["extend_rays"] + c["shadow_rays"]) / (frames + 1)
    ind.close()
    device.check()
    return {
        "scenes": count, "triangles_total": int(sum(tris)), "triangles_min": int(min(tris)),
        "triangles_max": int(max(tris)), "sites_total": int(sum(sites)), "sites_min": int(min(sites)),
        "sites_max": int(max(sites)), "samples_per_probe": samples_per_probe, "max_bounces": max_bounces,
        "scene_generation_s": generation_s, "setup_s": setup_s, "setup_workers": workers, "site_placement": dict(placement, method="the reference's adaptive weighted sample "
                                                                   "elimination on the GPU (density prepass, 5x "
                                                                   "oversampled candidates), no repair sites"),
        "autotune": tuned, "autotune_independent_samples": tuned_ind, "autotune_wavefront": tuned_wf,
        "autotune_wavefront_independent_samples": tuned_wfi,
        "ms_per_frame": {"per_scene_wavefront": per_scene_ms, "per_scene_megakernel": per_scene_mk_ms,
                         "batched": batch_ms, "batched_graph": graph_ms,
                         "batched_graph_wavefront": wf_ms,
                         "batched_graph_wavefront_independent_samples": wfi_ms,
                         "batched_graph_independent_samples": ind_ms},
        "rays_per_frame": batch_rays, "per_scene_rays_per_frame": per_scene_rays,
        "mrays_per_s": {"per_scene_wavefront": per_scene_rays / (per_scene_ms * 1e3),
                        "per_scene_megakernel": per_scene_rays / (per_scene_mk_ms * 1e3),
                        "batched": batch_rays / (batch_ms * 1e3), "batched_graph": batch_rays / (graph_ms * 1e3),
                        "batched_graph_wavefront": wf_rays / (wf_ms * 1e3),
                        "batched_graph_wavefront_independent_samples": wfi_rays / (wfi_ms * 1e3),
                        "batched_graph_independent_samples": ind_rays / (ind_ms * 1e3)},
    }


def main() -> None:
    """`--frames` batched frames over `--count` seeded scenes (no per-scene
    comparison); a small, self-contained workload for profiling."""
    import argparse

    import torch

    from nan_b200 import scenes as sc
    from nan_b200.probe_batch import ProbeBatch
    from nan_b200.render_data import RenderData
    from nan_b200.scene import Device, Scene
    from nan_b200.surface_probe_fields import SurfaceProbeRuntimeBuffers
    from nan_b200.surface_probe_path_tracer import SurfaceProbeDiffuseIrradianceBaker
    from nan_b200.surface_probe_resources import SurfaceProbeGpuGeometry

    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=16)
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--independent-samples", action="store_true")
    ap.add_argument("--wavefront", action="store_true")
    a = ap.parse_args()
    device = Device(0)
    items = []
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    sampler = SurfaceProbeSampler(device)
    for i, (node, n_sites) in enumerate(sc.batch_scenes(a.count, 1)):
        scene = Scene(device, node)
        geometry = SurfaceProbeGpuGeometry.create(
            device, SurfaceProbeSiteLayout.build_wse(node, n_sites, sampler=sampler, seed=1 + i,
                                                     repair_min_gather=0))
        baker = SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=64, max_bounces=3,
                                                   compensated=True)
        rt = SurfaceProbeRuntimeBuffers.acquire(RenderData(device), geometry.probe_count)
        items.append((scene, baker, rt.field, rt.attachments))
    batch = ProbeBatch(device, [(b, f, at) for _, b, f, at in items], independent_samples=a.independent_samples,
                       wavefront=a.wavefront)
    for f in range(a.frames):
        batch.execute(None, f, 64, 3, reset=(f == 0))
    torch.cuda.synchronize()
    device.check()
    print("ok", a.frames, "batched frames over", a.count, "scenes")


if __name__ == "__main__":
    main()
