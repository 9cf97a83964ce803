"""The wavefront's extend queue regrouped by ray direction octant
(NanTuning.ray_order = 1) changes only the order in which paths are traced:
texel slots, probe fields and screen pixels equal those of path order bit
for bit."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_ray_order_does_not_change_results(device):
    import torch

    import nan_b200
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout

    node = scenes.terrain_boxes(seed=3, grid=97, boxes=60)
    scene = nan_b200.Scene(device, node)
    layout = MeshColorsLayout.build(node, texels_per_unit=8.0, min_resolution=2, max_resolution=16)
    probes = nan_b200.SurfaceProbeSiteLayout.build(node, 2000, seed=2)
    geometry = nan_b200.SurfaceProbeGpuGeometry.create(device, probes)
    w, h = 64, 48
    node.camera.begin_frame(w, h)  # one jitter for both orders
    results = []
    for order in (0, 1):
        scene.configure("wavefront", ray_order=order)
        slots = torch.zeros((layout.total_payload_count, 4), dtype=torch.int32, device="cuda")
        tracer = nan_b200.TextureSpacePathTracer(device, scene, layout, samples_per_texel=2, max_bounces=3)
        for it in range(2):
            tracer.execute(None, slots, it, reset=(it == 0))
        rt = nan_b200.SurfaceProbeRuntimeBuffers.acquire(nan_b200.RenderData(device), probes.total_probe_count)
        baker = nan_b200.SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=8)
        for it in range(2):
            baker.execute(None, rt.field, rt.attachments, it, reset=(it == 0))
        out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
        nan_b200.PathTracer(device, scene).execute(None, out, 5)
        results.append([slots.clone(), rt.field.values.clone(), rt.attachments.radial_moments.clone(), out.clone()])
    scene.configure("wavefront")
    for a, b in zip(*results):
        torch.testing.assert_close(a, b, rtol=0, atol=0)
    device.check()
