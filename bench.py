#!/usr/bin/env python
"""Throughput of the texture-space (Mesh Colors) path-integration iteration.

Workload: one TextureSpacePathTracer iteration over every surface texel of a
seeded 200,688-triangle scene (313x313-vertex displaced terrain + 500 boxes
with sides U[0.2, 3] and random yaw, albedo U[0.1, 0.9]); 16 texels/unit,
per-triangle lattice resolution 4..64, 1 hemisphere sample per texel, 3
bounces, sun at 45 deg with irradiance 3, constant sky 0.5. One step = one
iteration (the wavefront integrator's generate/extend/shade/shadow/finalize
launches). Metric: Mrays/s, every closest-hit (extend) and any-hit (shadow)
ray counted on the device. The roofline is that of the traversal kernels
(k_wf_extend + k_wf_shadow), timed by CUDA events the library records on the
launching stream inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl nan|reference]

N > 1 runs under torchrun: each rank traces a contiguous 1/N range of the
surface texels (no data-path collective; strong scaling of a fixed frame).
``--impl reference`` times the reference's own CPU ray caster (tinybvh,
vertex_baker/cpp/tinybvh_visibility.cpp, built from the reference sources
into oracle/_ref/) on bounded samples of the same scene.
"""

from __future__ import annotations

import argparse
import gc
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = ("texture-space Mesh Colors iteration: seeded 200,688-triangle terrain (313x313 grid, "
            "height amplitude 2) + 500 boxes, 16 texels/unit, resolution 4-64, 1 sample/texel, 3 bounces")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["nan", "reference"], default="nan")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--grid", type=int, default=313)
    ap.add_argument("--boxes", type=int, default=500)
    ap.add_argument("--integrator", choices=["wavefront", "megakernel"], default="wavefront")
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="persistent traversal blocks per SM (0 = auto)")
    ap.add_argument("--bvh", choices=["sah", "ploc", "lbvh"], default="sah")
    ap.add_argument("--width", type=int, choices=[2, 8], default=2, help="traversed BVH node width")
    ap.add_argument("--paths", type=int, default=0, help="wavefront paths in flight (0 = one per texel)")
    ap.add_argument("--e2e-chunks", type=int, default=2,
                    help="texel chunks per e2e step (copies of one chunk overlap the tracing of the others)")
    ap.add_argument("--traversal", type=int, default=0, help="wavefront traversal form (NanTuning.traversal)")
    ap.add_argument("--ray-order", type=int, choices=[0, 1], default=0,
                    help="wavefront extend queue: 0 path order, 1 regrouped by direction octant")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-cache time-to-RMSE measurement")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-scene batched probe measurement")
    ap.add_argument("--no-cornell", action="store_true", help="skip the Cornell-box (area light) measurement")
    ap.add_argument("--no-city", action="store_true", help="skip the 4M-triangle city frame measurement")
    ap.add_argument("--no-consumers", action="store_true",
                    help="skip the resolve / filter / PRT / probe-resolve pass timings")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# Reference CPU caster (tinybvh) through ctypes.
# ---------------------------------------------------------------------------
VIS_SITES = 65536
VIS_RAYS = 512
VIS_DISTANCE = 1000.0
VIS_WORKLOAD = (f"PMR visibility SH: {VIS_SITES} seeded surface sites (seed 11) x {VIS_RAYS} rays of the reference "
                f"caster's direction table, self bias 1e-3, ray length {VIS_DISTANCE:g}, on the same world triangles")


def visibility_workload(node, world_triangles):
    """The one site set that the reference arm, the CPU baseline and the GPU
    visibility pass all trace: (positions, indices, sites, normals)."""
    from nan_b200 import scenes
    from oracle import visibility as ov

    positions, indices = ov.world_geometry(world_triangles)
    probes, _ = scenes.surface_sites(node, VIS_SITES, seed=11, double_sided_backs=False)
    return (positions, indices, np.ascontiguousarray(probes["position_radius"][:, :3]),
            np.ascontiguousarray(probes["normal_side"][:, :3]))


def cpu_baseline(workload):
    """The reference's own caster (tinybvh BVH8_CPU, all host threads) on the
    visibility site set: warm-up, then the median of 3 runs. Returns the
    cpu_baseline record and the caster's SH output."""
    from oracle import visibility as ov

    ref = ov.ReferenceCaster("bvh8")
    if not ref.available:
        return None, None
    positions, indices, sites, normals = workload
    ref.cast(positions, indices, sites, normals, VIS_RAYS, VIS_DISTANCE)
    runs = [ref.cast(positions, indices, sites, normals, VIS_RAYS, VIS_DISTANCE) for _ in range(3)]
    t = statistics.median(r[1]["trace_ms"] for r in runs)
    stats = runs[0][1]
    rays = sites.shape[0] * VIS_RAYS
    return ({"value": rays / (t * 1e3), "unit": "Mrays/s", "cores": stats["threads"], "kind": "reference",
             "sample": f"tinybvh {stats['layout']} any-hit ({stats['library']}): {VIS_WORKLOAD}; median of 3 runs "
                       f"({t:.0f} ms each), build {stats['build_ms']:.0f} ms, {os.cpu_count()} host cpus"},
            runs[0][0])


def pmr_visibility_line(scene, workload, reference_sh, steps=10):
    """GPU any-hit Mrays/s on exactly the CPU baseline's rays, and agreement
    with the reference caster's output (BVH8_CPU on every site; the scalar
    BVH layout, which runs the same watertight test, on the first 4096)."""
    import torch

    import nan_b200
    from oracle import visibility as ov

    positions, indices, sites, normals = workload
    dev = scene.device.torch_device
    sampler = nan_b200.PMRVisibilitySHSampler(scene.device)
    sites_d = torch.from_numpy(sites).to(dev)
    normals_d = torch.from_numpy(normals).to(dev)
    for _ in range(2):
        sh = sampler.sample(scene, sites_d, normals_d, ray_count=VIS_RAYS, max_distance=VIS_DISTANCE)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        sh = sampler.sample(scene, sites_d, normals_d, ray_count=VIS_RAYS, max_distance=VIS_DISTANCE)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    got = sh.cpu().numpy()
    rays = sites.shape[0] * VIS_RAYS
    out = {"workload": VIS_WORKLOAD, "sites": int(sites.shape[0]), "rays_per_site": VIS_RAYS,
           "gpu": {"ms": ms, "mrays_per_s": rays / (ms * 1e3), "kernel": "k_visibility_sh16"}}
    if reference_sh is not None:
        out["vs_reference_bvh8_cpu"] = ov.compare(reference_sh, got, VIS_RAYS)
    scalar = ov.ReferenceCaster("bvh")
    if scalar.available:
        k = 4096
        ref, _ = scalar.cast(positions, indices, sites[:k], normals[:k], VIS_RAYS, VIS_DISTANCE)
        out["vs_reference_bvh_first_4096"] = ov.compare(ref, got[:k], VIS_RAYS)
    return out


def roofline_bytes_per_ray(node, layout, lighting, sample_units: int = 6000):
    """Algorithmic bytes per ray = 32 + 16 + 32*N_node + 36*N_tri, with the node
    and triangle counts of the oracle's binned-SAH (8 bins) binary BVH on the
    same texel paths (sampled)."""
    from oracle.oracle import OracleScene

    orc = OracleScene(**node.pack())
    units = layout.units()
    rng = np.random.default_rng(3)
    pick = units[rng.choice(units.shape[0], size=min(sample_units, units.shape[0]), replace=False)]
    slots = np.zeros((layout.total_payload_count, 4), np.uint32)
    c = orc.trace_texels(lighting, slots, layout.face_array, layout.instance_array, layout.side_array, pick, 0, 1,
                         3, True)
    rays = c["extend_rays"] + c["shadow_rays"]
    n_node = c["node_fetches"] / rays
    n_tri = c["triangle_tests"] / rays
    roofline_bytes_per_ray.sah_cost = orc.bvh_stats()["sah_cost"]
    return 32.0 + 16.0 + 32.0 * n_node + 36.0 * n_tri, n_node, n_tri


def measured_peak_gbs():
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(peaks["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(integrator: str):
    """DRAM bytes (read + write) per step of the kernels the roofline covers,
    from the committed ncu summary."""
    try:
        data = json.loads((ROOT / "profiles" / "traffic.json").read_text())
        key = "traversal_bytes_per_step" if integrator == "wavefront" else "k_trace_texels_bytes_per_launch"
        return data.get(key)
    except Exception:
        return None


# ---------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from nan_b200 import scenes
    from oracle import visibility as ov
    from oracle.oracle import OracleScene

    ref = ov.ReferenceCaster("bvh8")
    if not ref.available:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref caster library not built"}))
        return
    node = scenes.terrain_boxes(seed=args.seed, grid=args.grid, boxes=args.boxes)
    positions, indices, sites, normals = visibility_workload(node, OracleScene(**node.pack()).world_triangles())
    for _ in range(max(args.warmup, 0)):
        ref.cast(positions, indices, sites, normals, VIS_RAYS, VIS_DISTANCE)
    total_ms, stats = 0.0, None
    for _ in range(args.steps):
        _, stats = ref.cast(positions, indices, sites, normals, VIS_RAYS, VIS_DISTANCE)
        total_ms += stats["trace_ms"]
    rays = args.steps * sites.shape[0] * VIS_RAYS
    value = rays / (total_ms * 1e3)
    line = {"impl": "reference", "metric": "Mrays/s", "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": WORKLOAD, "reference_step": VIS_WORKLOAD},
            "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": stats["threads"], "kind": "reference",
                             "sample": f"tinybvh {stats['layout']} ({stats['library']}): one step = {VIS_WORKLOAD}"},
            "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_nan(args):
    import torch
    import torch.distributed as dist

    import nan_b200
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout
    from nan_b200.parallel import shard_range

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    device = nan_b200.Device(local)
    node = scenes.terrain_boxes(seed=args.seed, grid=args.grid, boxes=args.boxes)
    scene = nan_b200.Scene(device, node, bvh_builder=args.bvh)
    layout = MeshColorsLayout.build(node, texels_per_unit=16.0, min_resolution=4, max_resolution=64)
    tracer = nan_b200.TextureSpacePathTracer(device, scene, layout, samples_per_texel=1, max_bounces=3,
                                             max_paths_in_flight=args.paths or None)
    scene.configure(args.integrator, trace_blocks_per_sm=args.blocks_per_sm, bvh_width=args.width,
                    ray_order=args.ray_order, traversal=args.traversal)
    total = layout.total_surface_texels
    begin, end = shard_range(total, rank, world)
    slots = torch.zeros((layout.total_payload_count, 4), dtype=torch.int32, device=device.torch_device)
    stream = torch.cuda.current_stream()

    it = 0
    for _ in range(args.warmup):
        tracer.execute(stream, slots, it, reset=(it == 0), texel_range=(begin, end))
        it += 1
    torch.cuda.synchronize()
    device.check()
    scene.context.read_counters(reset=True)
    launches0 = scene.context.launch_count
    # stage timing on inside the timed region: an event pair around each
    # wavefront launch, on the launching stream
    scene.configure(args.integrator, trace_blocks_per_sm=args.blocks_per_sm, bvh_width=args.width,
                    kernel_timing=True, ray_order=args.ray_order, traversal=args.traversal)
    scene.context.read_kernel_times(reset=True)

    clocks = ClockSampler(local)
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(args.steps):
        events[k][0].record(stream)
        tracer.execute(stream, slots, it, texel_range=(begin, end))
        events[k][1].record(stream)
        it += 1
    t1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clock_info = clocks.stop()
    elapsed_ms = t0.elapsed_time(t1)
    launch_ms = [a.elapsed_time(b) for a, b in events]
    launches = scene.context.launch_count - launches0
    counters = scene.context.read_counters(reset=True)
    ktimes = scene.context.read_kernel_times(reset=True)
    scene.configure(args.integrator, trace_blocks_per_sm=args.blocks_per_sm, bvh_width=args.width,
                    ray_order=args.ray_order, traversal=args.traversal)
    device.check()
    rays_local = counters["extend_rays"] + counters["shadow_rays"]

    # e2e through the public API with host buffers: every step the slot
    # buffer goes H2D from pinned memory, the iteration runs, and the updated
    # slots come back D2H (TextureSpacePathTracer.execute_host: per texel
    # chunk, so the copies of one chunk overlap the tracing of the others and
    # of the neighbouring steps; the timed region ends after the last copy).
    host_slots = torch.zeros_like(slots, device="cpu").pin_memory()
    host_slots.copy_(slots)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    tracer.execute_host(host_slots, slots, it, texel_range=(begin, end), chunks=args.e2e_chunks, stream=stream)
    tracer.host_ready(stream)
    it += 1
    barrier()
    torch.cuda.synchronize()
    scene.context.read_counters(reset=True)
    e0.record(stream)
    for k in range(args.steps):
        tracer.execute_host(host_slots, slots, it, texel_range=(begin, end), chunks=args.e2e_chunks, stream=stream)
        it += 1
    tracer.host_ready(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    e2e_counters = scene.context.read_counters(reset=True)
    e2e_rays_local = e2e_counters["extend_rays"] + e2e_counters["shadow_rays"]

    trav_ms = ktimes["extend_ms"] + ktimes["shadow_ms"]
    stats = torch.tensor([elapsed_ms, e2e_ms, trav_ms], dtype=torch.float64, device=device.torch_device)
    sums = torch.tensor([float(rays_local), float(e2e_rays_local)], dtype=torch.float64, device=device.torch_device)
    if world > 1:
        dist.all_reduce(stats, op=dist.ReduceOp.MAX)
        dist.all_reduce(sums, op=dist.ReduceOp.SUM)
    elapsed_ms, e2e_ms, trav_ms = float(stats[0]), float(stats[1]), float(stats[2])
    rays_total, e2e_rays = float(sums[0]), float(sums[1])
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return

    value = rays_total / (elapsed_ms * 1e3)
    bytes_per_ray, n_node, n_tri = roofline_bytes_per_ray(node, layout, scene.lighting)
    avg_step_s = statistics.mean(launch_ms) * 1e-3
    rays_per_step = rays_local / args.steps
    step_achieved = rays_per_step * bytes_per_ray / avg_step_s / 1e9
    if trav_ms > 0.0:
        # traversal kernels: all rays' algorithmic bytes over their own device time
        scope = "k_wf_extend + k_wf_shadow (per step: all extend and shadow launches)"
        achieved = rays_per_step * bytes_per_ray / (trav_ms / args.steps * 1e-3) / 1e9
    else:
        scope = "k_trace_texels (one launch per step)"
        achieved = step_achieved
    peak, peak_kind = measured_peak_gbs()
    traffic = ncu_traffic(args.integrator)
    line = {
        "metric": "Mrays/s", "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {
            "workload": WORKLOAD, "triangles": scene.triangle_count, "surface_texels": total,
            "payload_slots": layout.total_payload_count, "samples_per_texel": 1, "max_bounces": 3,
            "parallelism": f"texel-range shards x{world}" if world > 1 else "single GPU",
            "integrator": args.integrator,
            "bvh": args.bvh,
            "bvh_width": args.width,
            "l2": f"slot buffer {layout.total_payload_count * 16 / 1e6:.0f} MB read-modify-written per step "
                  "(> 126 MB L2)",
        },
        "rays_per_step": rays_total / args.steps,
        "extend_rays_per_step": counters["extend_rays"] / args.steps,
        "shadow_rays_per_step": counters["shadow_rays"] / args.steps,
        "bvh_build_ms": scene.info()["build_ms"],
        "bvh_sah_cost": scene.info()["sah_cost"],
        "reference_sah_cost": getattr(roofline_bytes_per_ray, "sah_cost", None),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "scope": scope,
                     "bytes_per_ray": bytes_per_ray, "nodes_per_ray": n_node, "tris_per_ray": n_tri,
                     "step_achieved": step_achieved, "step_frac": step_achieved / peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else peak_kind},
        "kernel_ms_per_step": {"extend": ktimes["extend_ms"] / args.steps, "shadow": ktimes["shadow_ms"] / args.steps,
                               "generate_shade_finalize": ktimes["stage_ms"] / args.steps},
        "e2e": {"value": e2e_rays / (e2e_ms * 1e3), "unit": "Mrays/s",
                "h2d_bytes_per_step": int(slots.numel() * 4), "d2h_bytes_per_step": int(slots.numel() * 4)},
        "gpu_launches": int(launches),
        "clocks": clock_info,
    }
    if world == 1 and not args.no_cpu_baseline:
        workload = visibility_workload(node, scene.world_triangles().cpu().numpy())
        line["cpu_baseline"], reference_sh = cpu_baseline(workload)
        line["pmr_visibility"] = pmr_visibility_line(scene, workload, reference_sh)
    if world == 1 and not args.no_learned:
        line["learned_cache"] = learned_cache_line(device)
    if world == 1 and not args.no_consumers:
        from benchmarks import consumers_eval

        line["consumers"] = consumers_eval.measure(device, scene, node, layout, slots, frames=5)
    if world == 1 and not args.no_cornell:
        line["cornell_area_light"] = cornell_line(device)
    if world == 1 and not args.no_city:
        from benchmarks import city_eval

        # start the 4M-triangle section from released memory: the earlier
        # sections' scenes and buffers otherwise stay cached
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        line["city_frame"] = city_eval.measure(device, frames=2)
    if world == 1 and not args.no_batched:
        from benchmarks import batch_eval

        line["batched_probes"] = dict(batch_eval.measure(device, count=64, seed=1, samples_per_probe=64,
                                                         max_bounces=3, frames=2),
                                      workload="64 seeded terrain+box scenes, triangles log-uniform 1e3-5e5, "
                                               "sites U{512..20480} per scene placed by the reference's adaptive "
                                               "weighted sample elimination of 5x oversampled candidates (no "
                                               "repair sites), 64 spp, 3 bounces, compensated running means")
    print(json.dumps(line))


def cornell_line(device) -> dict:
    """The 36-triangle Cornell box at 256x256, 16 frames of 1 spp, 3 bounces
    (4 path vertices): the reference's BSDF-only path tracer against the
    area-light NEE + MIS option, each scored by relative RMSE against 4096
    BSDF-only frames accumulated in float64."""
    import torch

    import nan_b200
    from nan_b200 import scenes

    node = scenes.cornell_box(256, 256)
    scene = nan_b200.Scene(device, node)
    scene.enable_area_lights()
    tracer = nan_b200.PathTracer(device, scene, max_vertices=4)
    w = h = 256
    out = torch.zeros((h, w, 4), dtype=torch.float32, device=device.torch_device)
    stream = torch.cuda.current_stream()

    def run(area, frames, base, timed=False):
        scene.lighting.area_nee = area
        acc = torch.zeros((h, w, 3), dtype=torch.float64, device=device.torch_device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = 0.0
        for f in range(frames):
            node.camera.begin_frame(w, h)
            e0.record(stream)
            tracer.execute(stream, out, base + f)
            e1.record(stream)
            acc += out[..., :3].double()
            if timed:
                e1.synchronize()
                ms += e0.elapsed_time(e1)
        return acc / frames, ms

    ref, _ = run(False, 4096, 1_000_000)
    res = {"scene": "Cornell box, 36 triangles, light quad emission (17, 12, 4)", "image": "256x256",
           "frames": 16, "max_vertices": 4, "reference_frames": 4096}
    for name, area in (("bsdf_only", False), ("area_nee_mis", True)):
        run(area, 4, 50_000)  # warm-up
        img, ms = run(area, 16, 0, timed=True)
        rmse = float(torch.sqrt(torch.mean((img - ref) ** 2)) / torch.sqrt(torch.mean(ref ** 2)))
        res[name] = {"ms_per_frame": ms / 16, "relative_rmse": rmse}
    scene.lighting.area_nee = False
    return res


def learned_cache_line(device) -> dict:
    """Time to RMSE of the learned-cache path tracer against the plain one on
    the seeded 998,408-triangle scene (699x699 terrain + 2000 boxes) at
    1920x1080, 1 spp per frame, against a 256-frame plain reference
    accumulated in float64."""
    import torch

    import nan_b200
    from benchmarks import learned_eval
    from nan_b200 import scenes

    node = scenes.terrain_boxes(seed=1, grid=699, boxes=2000)
    scene = nan_b200.Scene(device, node)
    out = {"scene": f"terrain 699x699 + 2000 boxes, {scene.triangle_count} triangles, sun 45 deg + sky 0.5",
           "image": "1920x1080, 1 spp per frame, 5 path vertices", "runs": []}
    # 8 warm-up frames: a sweep of 0-32 put the time to the target lowest near 6-8 (32 frames
    # cost 113 ms up front; fewer than 6 leave the cache above the RMSE bar after 64 frames)
    warmup = 8
    for cv, batch in ((1, 16384), (0, 8192)):
        r = learned_eval.compare(device, scene, 1920, 1080, reference_frames=256, frames=64, cache_vertex=cv,
                                 warmup_frames=warmup, train_batch=batch, table_update="lazy")
        out["runs"].append({
            "cache_vertex": cv, "warmup_frames": warmup, "train_samples_per_frame": 65536, "train_batch": batch,
            "table_update": "lazy Adam (touched entries only)",
            "frontier": [{k: (round(v, 5) if isinstance(v, float) else v) for k, v in f.items()}
                         for f in r["frontier"]],
            "target_rmse": r["target_rmse"], "plain_ms_to_target": r["plain_ms_to_target"],
            "cached_ms_to_target": r["cached_ms_to_target"], "speedup": r["speedup"],
            "rmse_after_64_frames": r["rmse_per_frame_count"],
            "ms_per_frame": {"plain": r["plain_ms_per_frame"], "cached": r["cached_ms_per_frame"],
                             "cached_without_training": r["untrained_ms_per_frame"]},
            "cached_warmup_ms": r["cached_warmup_ms"],
            "cached_curve": [[n, round(ms, 2), round(e, 5)] for n, ms, e in r["cached"]
                             if n in (1, 2, 4, 8, 12, 16, 24, 32, 48, 64)],
            "plain_curve": [[n, round(ms, 2), round(e, 5)] for n, ms, e in r["plain"]],
        })
        del r
    torch.cuda.synchronize()
    return out


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_nan(args)


if __name__ == "__main__":
    main()
