"""Time to a target RMSE: the plain screen path tracer against the same path
tracer with the learned radiance cache, on one scene.

The reference image is the plain path tracer (max_vertices path vertices)
accumulated over many frames in float64 on the GPU (FP64 is used only for
this reduction). Both integrators start cold and accumulate 1 spp frames;
the learned one first renders `warmup_frames` frames that only train the
cache (their time counts, their images are not accumulated). Every frame is
timed with CUDA events on the launching stream (render, plus the cache's
training for the learned integrator). The error of an accumulated image is
its relative RMSE against the reference over all pixels and channels.
"""

from __future__ import annotations

from nan_b200.radiance_cache import scene_bounds


def _rel_rmse(img, ref) -> float:
    import torch

    d = img - ref
    return float(torch.sqrt(torch.mean(d * d)) / torch.sqrt(torch.mean(ref * ref)))


def compare(device, scene, width: int, height: int, *, reference_frames: int = 512, frames: int = 64,
            max_vertices: int = 5, train_samples: int = 65536, train_batch: int = 65536, log2_table: int = 19,
            base_resolution: int = 16, max_resolution: int = 2048, learning_rate: float = 1e-2,
            checkpoints=None, seed: int = 0, cache_vertex: int = 1, warmup_frames: int = 0,
            table_update: str = "dense", lr_decay: float = 1.0, lr_min: float = 0.0,
            train_frames: int | None = None) -> dict:
    """Curves (frames, cumulative ms, relative RMSE) of the plain and the
    cached integrator, and the time each needs to reach the plain
    integrator's RMSE after `frames` frames (within 1.1x for the cached one).

    Training schedule of the cached integrator: the learning rate of
    training frame f (warm-up frames first) is max(learning_rate *
    lr_decay**f, lr_min); after `train_frames` training frames (None: all)
    the cache is frozen and frames only render. `frontier` lists, for every
    plain checkpoint k, the time each integrator needs to reach the plain
    RMSE after k frames (1.1x for the cached one)."""
    import torch

    from nan_b200.cached_path_tracer import CachedPathTracer
    from nan_b200.path_tracer import PathTracer
    from nan_b200.radiance_cache import RadianceCache

    stream = torch.cuda.current_stream()
    cam = scene.camera
    out = torch.zeros((height, width, 4), dtype=torch.float32, device=device.torch_device)
    plain = PathTracer(device, scene, max_vertices=max_vertices)

    ref = torch.zeros((height, width, 3), dtype=torch.float64, device=device.torch_device)
    for f in range(reference_frames):
        cam.begin_frame(width, height)
        plain.execute(stream, out, 1_000_000 + f)
        ref += out[..., :3].double()
    ref /= reference_frames

    checkpoints = sorted(set(checkpoints or [1, 2, 4, 8, 16, 32, 64, 128, 256]))
    checkpoints = [c for c in checkpoints if c <= frames] or [frames]
    if checkpoints[-1] != frames:
        checkpoints.append(frames)

    warm_ms = {}

    def schedule(tracer, f):
        if not hasattr(tracer, "cache") or not getattr(tracer, "_schedule", False):
            return
        if train_frames is not None and f >= train_frames:
            tracer.train = False
        else:
            tracer.cache.set_learning_rate(max(learning_rate * lr_decay ** f, lr_min))

    def run(tracer, warmup=0, every=None) -> list[tuple[int, float, float]]:
        acc = torch.zeros((height, width, 3), dtype=torch.float64, device=device.torch_device)
        curve, total_ms = [], 0.0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for f in range(warmup):
            schedule(tracer, f)
            cam.begin_frame(width, height)
            e0.record(stream)
            tracer.execute(stream, out, frames + f)
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
        warm_ms[id(tracer)] = total_ms
        for f in range(frames):
            schedule(tracer, warmup + f)
            cam.begin_frame(width, height)
            e0.record(stream)
            tracer.execute(stream, out, f)
            e1.record(stream)
            acc += out[..., :3].double()
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            if f + 1 in checkpoints or (every and (f + 1) % every == 0):
                curve.append((f + 1, total_ms, _rel_rmse(acc / (f + 1), ref)))
        return curve

    plain_curve = run(plain)
    lo, hi = scene_bounds(scene)
    cache = RadianceCache(device, lo, hi, log2_table=log2_table, base_resolution=base_resolution,
                          max_resolution=max_resolution, learning_rate=learning_rate, seed=seed,
                          table_update=table_update)
    cached = CachedPathTracer(device, scene, cache, cache_vertex=cache_vertex, max_vertices=max_vertices,
                              train_samples=train_samples, train_batch=train_batch)
    cached._schedule = True
    cached_curve = run(cached, warmup_frames, every=1)
    cached_warm_ms = warm_ms[id(cached)]
    # the same cached integrator with the cache left untrained: what training gains
    cold = RadianceCache(device, lo, hi, log2_table=log2_table, base_resolution=base_resolution,
                         max_resolution=max_resolution, seed=seed)
    untrained_curve = run(CachedPathTracer(device, scene, cold, cache_vertex=cache_vertex, max_vertices=max_vertices,
                                           train=False))

    target = plain_curve[-1][2]
    t_plain = plain_curve[-1][1]
    t_cached = next((ms for (_, ms, e) in cached_curve if e <= 1.1 * target), None)
    frontier = []
    for k, ms_p, e_p in plain_curve:
        ms_c = next((ms for (_, ms, e) in cached_curve if e <= 1.1 * e_p), None)
        frontier.append({"plain_frames": k, "target_rmse": e_p, "plain_ms": ms_p, "cached_ms": ms_c,
                         "speedup": (ms_p / ms_c) if ms_c else None})
    device.check()
    return {
        "width": width, "height": height, "frames": frames, "reference_frames": reference_frames,
        "max_vertices": max_vertices, "train_samples": train_samples, "train_batch": train_batch,
        "cache_vertex": cache_vertex, "warmup_frames": warmup_frames,
        "plain": plain_curve, "cached": cached_curve, "untrained": untrained_curve,
        "target_rmse": target, "plain_ms_to_target": t_plain, "cached_ms_to_target": t_cached,
        "speedup": (t_plain / t_cached) if t_cached else None, "frontier": frontier,
        "schedule": {"table_update": table_update, "learning_rate": learning_rate, "lr_decay": lr_decay,
                     "lr_min": lr_min, "train_frames": train_frames},
        "plain_ms_per_frame": plain_curve[-1][1] / frames,
        "cached_ms_per_frame": (cached_curve[-1][1] - cached_warm_ms) / frames, "cached_warmup_ms": cached_warm_ms,
        "untrained_ms_per_frame": untrained_curve[-1][1] / frames,
        "rmse_per_frame_count": {"plain": plain_curve[-1][2], "cached": cached_curve[-1][2],
                                 "untrained": untrained_curve[-1][2]},
    }


def summary(r: dict) -> str:
    lines = [f"{r['width']}x{r['height']}, cache vertex {r['cache_vertex']}, warm-up {r['warmup_frames']}, reference "
             f"{r['reference_frames']} frames, target = plain RMSE after {r['frames']} frames = {r['target_rmse']:.4f}"]
    for name in ("plain", "cached", "untrained"):
        lines.append(name + ": " + ", ".join(f"{n}f {ms:.0f}ms {e:.4f}" for n, ms, e in r[name]))
    sp = r["speedup"]
    lines.append(f"time to target: plain {r['plain_ms_to_target']:.0f} ms, cached "
                 f"{r['cached_ms_to_target'] if r['cached_ms_to_target'] is None else round(r['cached_ms_to_target'])}"
                 f" ms, speed-up {'n/a' if sp is None else f'{sp:.2f}x'}")
    return "\n".join(lines)


__all__ = ["compare", "summary", "scene_bounds"]


def main() -> None:
    """Run `--frames` cached frames (render + online training) on the seeded
    998,408-triangle scene; a small, self-contained workload for profiling."""
    import argparse

    import torch

    from nan_b200 import scenes
    from nan_b200.cached_path_tracer import CachedPathTracer
    from nan_b200.radiance_cache import RadianceCache
    from nan_b200.scene import Device, Scene

    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=6)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--cache-vertex", type=int, default=1)
    ap.add_argument("--table-update", choices=("dense", "lazy"), default="lazy",
                    help="Adam over the whole hash table or only the entries a step touched (the bench's)")
    a = ap.parse_args()
    device = Device(0)
    node = scenes.terrain_boxes(seed=1, grid=699, boxes=2000)
    scene = Scene(device, node)
    lo, hi = scene_bounds(scene)
    tracer = CachedPathTracer(device, scene, RadianceCache(device, lo, hi, table_update=a.table_update),
                              cache_vertex=a.cache_vertex, train_batch=16384)
    out = torch.zeros((a.height, a.width, 4), dtype=torch.float32, device=device.torch_device)
    for f in range(a.frames):
        node.camera.begin_frame(a.width, a.height)
        tracer.execute(None, out, f)
    torch.cuda.synchronize()
    device.check()
    print("ok", a.frames, "cached frames")


if __name__ == "__main__":
    main()
