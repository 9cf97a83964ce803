"""Precision of the accumulated results (GPU required).

* Compensated running means: over 300-400 iterations the Kahan-compensated
  means stay within 5e-7 (relative) of the FP64 mean of the same per-iteration
  samples and are at least 4x closer on average than the reference's plain
  lerp (measured on B200: 1.3e-7 max vs 1.5e-6 for lerp).
* FP64 oracle: converged texel caches (24 iterations) and a 16-frame screen
  image from the FP32 CUDA path against the oracle evaluated in double
  precision on the same RNG streams. Stated bound: relative RMSE <= 1e-5 and
  >= 99.9 % of values within 1e-4 (measured: 1.2e-7 and 2.5e-8 RMSE).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cornell(device):
    import nan_b200
    from nan_b200 import scenes

    node = scenes.cornell_box(48, 48)
    return node, nan_b200.Scene(device, node)


def test_compensated_texel_means_track_fp64(device):
    import torch

    import nan_b200
    from nan_b200.mesh_colors import MeshColorsLayout

    node, scene = _cornell(device)
    layout = MeshColorsLayout.build(node, texels_per_unit=6.0, min_resolution=2, max_resolution=8)
    P = layout.total_payload_count
    plain = nan_b200.TextureSpacePathTracer(device, scene, layout, max_bounces=3)
    comp = nan_b200.TextureSpacePathTracer(device, scene, layout, max_bounces=3, compensated=True)
    probe = nan_b200.TextureSpacePathTracer(device, scene, layout, max_bounces=3)
    slots_a = torch.zeros((P, 4), dtype=torch.int32, device="cuda")
    slots_b = torch.zeros_like(slots_a)
    sample = torch.zeros_like(slots_a)
    mean64 = np.zeros((P, 3), np.float64)
    n = 400
    for it in range(n):
        plain.execute(None, slots_a, it, reset=(it == 0))
        comp.execute(None, slots_b, it, reset=(it == 0))
        probe.execute(None, sample, it, reset=True)  # this iteration's sample itself
        mean64 += sample.cpu().numpy().view(np.float32)[:, :3].astype(np.float64)
    mean64 /= n
    a = slots_a.cpu().numpy().view(np.float32)[:, :3].astype(np.float64)
    b = slots_b.cpu().numpy().view(np.float32)[:, :3].astype(np.float64)
    assert np.all(slots_b.cpu().numpy()[:, 3] == n)
    scale = np.maximum(np.abs(mean64), 1e-3)
    err_a = np.abs(a - mean64) / scale
    err_b = np.abs(b - mean64) / scale
    print("texel means: plain max/mean", err_a.max(), err_a.mean(), "compensated", err_b.max(), err_b.mean())
    assert err_b.max() <= 5e-7, err_b.max()
    assert err_b.mean() <= 0.25 * err_a.mean(), (err_b.mean(), err_a.mean())
    device.check()


def test_compensated_probe_means_track_fp64(device):
    import torch

    import nan_b200
    from nan_b200 import scenes

    node, scene = _cornell(device)
    probes, pinst = scenes.surface_sites(node, 400, seed=5, radius=0.2)
    layout = type("L", (), {})()
    layout.probes, layout.instance_gpu_data = probes, pinst
    layout.nodes = np.zeros((1, 4), np.uint32)
    layout.triangle_vertex_probes = np.zeros((1, 4), np.uint32)
    layout.total_probe_count = probes.shape[0]
    layout.instance_infos = list(range(pinst.shape[0]))
    geometry = nan_b200.SurfaceProbeGpuGeometry.create(device, layout)
    n = probes.shape[0]
    bakers = [nan_b200.SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=4,
                                                          compensated=c) for c in (False, True, False)]
    buffers = [nan_b200.SurfaceProbeRuntimeBuffers.acquire(nan_b200.RenderData(device), n) for _ in range(3)]
    mean64 = np.zeros((n, 3), np.float64)
    iters = 300
    for it in range(iters):
        for k in range(3):
            bakers[k].execute(None, buffers[k].field, buffers[k].attachments, it, reset=(it == 0 or k == 2))
        mean64 += buffers[2].field.values.cpu().numpy().view(np.float32).reshape(n, 3).astype(np.float64)
    mean64 /= iters
    a = buffers[0].field.values.cpu().numpy().view(np.float32).reshape(n, 3).astype(np.float64)
    b = buffers[1].field.values.cpu().numpy().view(np.float32).reshape(n, 3).astype(np.float64)
    scale = np.maximum(np.abs(mean64), 1e-3)
    err_a = np.abs(a - mean64) / scale
    err_b = np.abs(b - mean64) / scale
    print("probe means: plain max/mean", err_a.max(), err_a.mean(), "compensated", err_b.max(), err_b.mean())
    assert err_b.max() <= 5e-7, err_b.max()
    assert err_b.mean() <= 0.25 * err_a.mean()
    device.check()


def test_converged_texels_and_image_vs_fp64_oracle(device):
    import torch

    import nan_b200
    from nan_b200.mesh_colors import MeshColorsLayout
    from oracle.oracle import F64, OracleScene

    node, scene = _cornell(device)
    orc = OracleScene(**scene.host)
    layout = MeshColorsLayout.build(node, texels_per_unit=6.0, min_resolution=2, max_resolution=8)
    tracer = nan_b200.TextureSpacePathTracer(device, scene, layout, max_bounces=3)
    slots = torch.zeros((layout.total_payload_count, 4), dtype=torch.int32, device="cuda")
    units = layout.units()[::7]
    host = np.zeros((layout.total_payload_count, 4), np.uint32)
    iters = 24
    for it in range(iters):
        tracer.execute(None, slots, it, reset=(it == 0))
        orc.trace_texels(scene.lighting, host, layout.face_array, layout.instance_array, layout.side_array, units,
                         it, 1, 3, it == 0, precision=F64)
    front = layout.instance_array[units[:, 0], 2] + units[:, 1]
    g = slots.cpu().numpy().view(np.float32)[front, :3].astype(np.float64)
    o = host.view(np.float32)[front, :3].astype(np.float64)
    rel_rmse = np.sqrt(np.mean((g - o) ** 2)) / max(np.sqrt(np.mean(o**2)), 1e-12)
    close = np.all(np.abs(g - o) <= 1e-4 * np.maximum(np.abs(o), 1e-2), axis=1).mean()
    print("texels vs FP64 oracle: rel RMSE", rel_rmse, "within 1e-4:", close)
    assert close >= 0.999 and rel_rmse <= 1e-5, (close, rel_rmse)

    # screen: 16 accumulated frames of the path tracer vs the FP64 oracle
    w = h = 48
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    disp = torch.zeros_like(out)
    rd = nan_b200.RenderData(device)
    acc = nan_b200.Accumulator(device)
    pt = nan_b200.PathTracer(device, scene)
    px = np.stack(np.meshgrid(np.arange(w), np.arange(h), indexing="xy"), -1).reshape(-1, 2)
    ref = np.zeros((w * h, 3), np.float64)
    cam = node.camera
    for frame in range(16):
        cam.begin_frame(w, h)
        pt.execute(None, out, frame)
        acc.execute(None, rd, out, disp, reset=(frame == 0))
        r, _ = orc.trace_screen(scene.lighting, cam, w, h, frame, 5, px, precision=F64)
        ref += r[:, :3].astype(np.float64)
    ref /= 16
    img = disp.cpu().numpy().reshape(-1, 4)[:, :3].astype(np.float64)
    rel_rmse = np.sqrt(np.mean((img - ref) ** 2)) / max(np.sqrt(np.mean(ref**2)), 1e-12)
    close = np.all(np.abs(img - ref) <= 1e-4 * np.maximum(np.abs(ref), 1e-2), axis=1).mean()
    print("image vs FP64 oracle: rel RMSE", rel_rmse, "within 1e-4:", close)
    assert close >= 0.999 and rel_rmse <= 1e-5, (close, rel_rmse)
    device.check()
