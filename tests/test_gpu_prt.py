"""PRT L2 baker and evaluator on the GPU against the oracle, on the terrain
and on the Cornell box (emissive ceiling, sun): after three iterations the
transport, static source, self hits and radial moments equal the oracle's
bit for bit for >= 99.9 % of probes (counts always); the lighting projection
and the evaluated field equal the oracle's bit for bit."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["terrain", "cornell"])
def test_prt_baker_and_evaluator_match_oracle(which, device):
    import nan_b200
    from nan_b200 import scenes
    from nan_b200.surface_probe_fields import (DIFFUSE_PRT_ATTACHMENTS, DIFFUSE_PRT_L2_RGB_FIELD,
                                               SurfaceProbeRuntimeBuffers)
    from oracle.oracle import OracleScene, prt_evaluate, prt_project_lighting

    if which == "terrain":
        node = scenes.terrain_boxes(seed=1, grid=129, boxes=120)
        node.lighting.sky_radiance = (0.4, 0.5, 0.7)
    else:
        node = scenes.cornell_box(32, 32)
        node.lighting.sky_radiance = (0.2, 0.2, 0.3)
    scene = nan_b200.Scene(device, node)
    orc = OracleScene(**scene.host)
    probes, pinst = scenes.surface_sites(node, 1500, seed=5, radius=0.3)
    layout = type("L", (), {})()
    layout.probes = probes
    layout.nodes = np.zeros((1, 4), np.uint32)
    layout.instance_gpu_data = pinst
    layout.triangle_vertex_probes = np.zeros((1, 4), np.uint32)
    layout.total_probe_count = probes.shape[0]
    layout.instance_infos = list(range(pinst.shape[0]))
    geometry = nan_b200.SurfaceProbeGpuGeometry.create(device, layout)
    rd = nan_b200.RenderData(device)
    rt = SurfaceProbeRuntimeBuffers.acquire(rd, probes.shape[0], field_desc=DIFFUSE_PRT_L2_RGB_FIELD,
                                            attachment_descs=DIFFUSE_PRT_ATTACHMENTS)
    baker = nan_b200.SurfaceProbePrtBaker(device, scene, geometry, samples_per_probe=8, max_bounces=3)
    with pytest.raises(ValueError):
        baker.execute(None, SurfaceProbeRuntimeBuffers.acquire(rd, probes.shape[0]).field, rt.attachments, 0)
    n = probes.shape[0]
    values = np.zeros((n, 27), np.float32)
    counts = np.zeros(n, np.uint32)
    self_hits = np.zeros(n, np.uint32)
    radial = np.zeros((n, 16), np.uint32)
    static = np.zeros((n, 3), np.float32)
    for it in range(3):
        baker.execute(None, rt.field, rt.attachments, it, reset=(it == 0))
        orc.trace_probes_prt(scene.lighting, values, counts, self_hits, radial, static, probes, pinst,
                             np.arange(n, dtype=np.uint32), it, 8, 3, it == 0)
    g_values = rt.field.values.cpu().numpy().view(np.float32).reshape(n, 27)
    g_counts = rt.field.sample_counts.cpu().numpy().view(np.uint32)
    g_self = rt.attachments.self_hit_counts.cpu().numpy().view(np.uint32)
    g_radial = rt.attachments.radial_moments.cpu().numpy().view(np.uint32).reshape(n, 16)
    g_static = rt.attachments.static_source_rgb.cpu().numpy().view(np.float32).reshape(n, 3)
    np.testing.assert_array_equal(g_counts, counts)
    exact = (np.all(g_values == values, axis=1) & np.all(g_static == static, axis=1) & (g_self == self_hits)
             & np.all(g_radial == radial, axis=1))
    print(which, "probes", n, "exact", exact.mean(), "static > 0", (static.sum(1) > 0).mean())
    assert exact.mean() >= 0.999, exact.mean()
    assert np.abs(values).max() > 0

    evaluator = nan_b200.SurfaceProbePrtEvaluator(device, scene, geometry)
    evaluated = evaluator.execute(None, rd, rt.field, rt.attachments)
    g_sh = rd.get_buffer("surface_probe_renderer.prt.lighting_sh", struct_size=16, element_count=9)
    g_sh = g_sh.cpu().numpy().view(np.float32).reshape(9, 4)
    sh = prt_project_lighting(scene.lighting, evaluator.LIGHTING_PROJECTION_SAMPLE_COUNT)
    np.testing.assert_array_equal(g_sh, sh)
    out, out_counts = prt_evaluate(g_values, g_counts, g_static, sh)
    np.testing.assert_array_equal(evaluated.values.cpu().numpy().view(np.float32).reshape(n, 3), out)
    np.testing.assert_array_equal(evaluated.sample_counts.cpu().numpy().view(np.uint32), out_counts)
    assert out.max() > 0
    device.check()
