"""Surface-probe resolve on the GPU against the oracle: probes placed by
SurfaceProbeSiteLayout (per-instance point octrees), an irradiance field
baked on the GPU, then the beauty view (with and without the radial
visibility prior) and debug views 1-5 equal the oracle's resolve of the same
field bit for bit on >= 99.9 % of pixels, on the terrain and the Cornell
box."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["terrain", "cornell"])
def test_probe_resolve_matches_oracle(which, device):
    import torch

    import nan_b200
    from nan_b200 import scenes
    from oracle.oracle import OracleScene

    if which == "terrain":
        node = scenes.terrain_boxes(seed=1, grid=129, boxes=120)
        node.lighting.sky_radiance = (0.3, 0.4, 0.6)
        sites = 6000
    else:
        node = scenes.cornell_box(64, 64)
        sites = 3000
    scene = nan_b200.Scene(device, node)
    orc = OracleScene(**scene.host)
    layout = nan_b200.SurfaceProbeSiteLayout.build(node, sites, seed=7)
    geometry = nan_b200.SurfaceProbeGpuGeometry.create(device, layout)
    rd = nan_b200.RenderData(device)
    rt = nan_b200.SurfaceProbeRuntimeBuffers.acquire(rd, layout.total_probe_count)
    baker = nan_b200.SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=16, max_bounces=3)
    for it in range(4):
        baker.execute(None, rt.field, rt.attachments, it, reset=(it == 0))
    n = layout.total_probe_count
    values = rt.field.values.cpu().numpy().view(np.float32).reshape(n, 3)
    counts = rt.field.sample_counts.cpu().numpy().view(np.uint32)
    self_hits = rt.attachments.self_hit_counts.cpu().numpy().view(np.uint32)
    radial = rt.attachments.radial_moments.cpu().numpy().view(np.uint32).reshape(n, 16)
    assert counts.min() == 4 and np.any(radial != 0)

    resolve = nan_b200.SurfaceProbeResolve(device, scene, layout, geometry)
    w, h = 96, 64
    node.camera.begin_frame(w, h)
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    px = np.stack(np.meshgrid(np.arange(w), np.arange(h), indexing="xy"), -1).reshape(-1, 2)
    cases = [dict(debug_view=0), dict(debug_view=0, use_radial_visibility=False),
             dict(debug_view=0, min_gather_count=24)] + [dict(debug_view=v) for v in range(1, 6)]
    for kw in cases:
        resolve.execute(None, rt.field, rt.attachments, out, **kw)
        gpu = out.cpu().numpy().reshape(-1, 4)
        ref = orc.resolve_probes(scene.lighting, node.camera, w, h, px, layout, values, counts, self_hits, radial,
                                 frame_index=scene.frame_index, **kw)
        exact = np.all(gpu == ref, axis=1)
        rel = np.max(np.abs(gpu - ref) / np.maximum(np.abs(ref), 1e-3), axis=1)
        print(which, kw, "exact", exact.mean(), "max rel", rel.max())
        assert exact.mean() >= 0.999, (kw, exact.mean())
        assert (rel <= 1e-4).mean() >= 0.999
    device.check()


def test_vertex_anchor_fallback_matches_oracle(device):
    """build_vertex_anchors: one anchor probe per render vertex (both sides
    on the double-sided walls), outside the octree, and a triangle map the
    resolve's vertex fallback reads; with few sites and min gather 24 the
    fallback blends in, and GPU and oracle agree as above."""
    import torch

    import nan_b200
    from nan_b200 import scenes
    from nan_b200.surface_probe_resources import SURFACE_PROBE_FLAG_VERTEX_ANCHOR
    from oracle.oracle import OracleScene

    node = scenes.reference_demo()
    scene = nan_b200.Scene(device, node)
    orc = OracleScene(**scene.host)
    layout = nan_b200.SurfaceProbeSiteLayout.build_wse(node, 60, seed=3, build_vertex_anchors=True, device=device)
    anchor = (layout.probes["meta"][:, 3] & SURFACE_PROBE_FLAG_VERTEX_ANCHOR) != 0
    expected = 0
    for i, (mesh_id, mat_id, _) in enumerate(node.instances):
        sides = 2 if node.materials[mat_id].double_sided else 1
        expected += sides * np.unique(node.meshes[mesh_id].indices).shape[0]
    assert int(anchor.sum()) == expected
    # anchors sit after each instance's octree-ordered probes, outside its octree
    for i, info in enumerate(layout.instance_infos):
        found = layout.query_probe_indices(i, info.root_center, radius=info.root_extent * 4.0)
        assert not anchor[found].any()
        assert found.shape[0] == info.reconstruction_probe_count
    maps = layout.triangle_vertex_probes
    valid = (maps[:, 3] & 1) != 0
    assert valid.any() and np.all(anchor[maps[valid, :3].reshape(-1)])

    geometry = nan_b200.SurfaceProbeGpuGeometry.create(device, layout)
    rd = nan_b200.RenderData(device)
    rt = nan_b200.SurfaceProbeRuntimeBuffers.acquire(rd, layout.total_probe_count)
    baker = nan_b200.SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=16, max_bounces=3)
    for it in range(2):
        baker.execute(None, rt.field, rt.attachments, it, reset=(it == 0))
    n = layout.total_probe_count
    values = rt.field.values.cpu().numpy().view(np.float32).reshape(n, 3)
    counts = rt.field.sample_counts.cpu().numpy().view(np.uint32)
    self_hits = rt.attachments.self_hit_counts.cpu().numpy().view(np.uint32)
    radial = rt.attachments.radial_moments.cpu().numpy().view(np.uint32).reshape(n, 16)
    resolve = nan_b200.SurfaceProbeResolve(device, scene, layout, geometry)
    w, h = 96, 64
    node.camera.begin_frame(w, h)
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    px = np.stack(np.meshgrid(np.arange(w), np.arange(h), indexing="xy"), -1).reshape(-1, 2)
    plain = None
    for kw in (dict(debug_view=0), dict(debug_view=0, use_vertex_fallback=True),
               dict(debug_view=0, use_vertex_fallback=True, min_gather_count=24)):
        resolve.execute(None, rt.field, rt.attachments, out, **kw)
        gpu = out.cpu().numpy().reshape(-1, 4)
        ref = orc.resolve_probes(scene.lighting, node.camera, w, h, px, layout, values, counts, self_hits, radial,
                                 frame_index=scene.frame_index, **kw)
        exact = np.all(gpu == ref, axis=1)
        print("anchors", kw, "exact", exact.mean())
        assert exact.mean() >= 0.999, (kw, exact.mean())
        if plain is None:
            plain = gpu
        elif kw.get("min_gather_count") == 24:
            assert np.any(gpu != plain)  # the fallback changes pixels where confidence is low
    device.check()
