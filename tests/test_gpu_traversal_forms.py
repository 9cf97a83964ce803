"""Every wavefront traversal form (NanTuning.traversal: whole-warp ray
grabs, lanes refilled from the queue at several thresholds, a shared-memory
stack top, the speculative while-while walk) changes only
which lane walks which ray and when: texel slots, probe fields, screen
pixels and the ray counts equal those of the default form bit for bit, on
PLOC and LBVH trees (LBVH leaves hold up to 8 triangles)."""

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("builder", ["sah", "ploc", "lbvh"])
def test_traversal_forms_do_not_change_results(device, builder):
    import torch

    import nan_b200
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout

    node = scenes.terrain_boxes(seed=5, grid=97, boxes=60)
    scene = nan_b200.Scene(device, node, bvh_builder=builder)
    layout = MeshColorsLayout.build(node, texels_per_unit=8.0, min_resolution=2, max_resolution=16)
    probes = nan_b200.SurfaceProbeSiteLayout.build(node, 2000, seed=2)
    geometry = nan_b200.SurfaceProbeGpuGeometry.create(device, probes)
    w, h = 64, 48
    node.camera.begin_frame(w, h)
    results, rays = [], []
    for form in (0, 1, 2, 3, 4, 5, 6):
        scene.configure("wavefront", traversal=form)
        scene.context.read_counters(reset=True)
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
        c = scene.context.read_counters(reset=True)
        rays.append((c["extend_rays"], c["shadow_rays"]))
    scene.configure("wavefront")
    for other in results[1:]:
        for a, b in zip(results[0], other):
            torch.testing.assert_close(a, b, rtol=0, atol=0)
    assert all(r == rays[0] for r in rays)
    device.check()
