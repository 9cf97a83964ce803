"""Sky-view LUT on the GPU: with a seeded 200x200 RGBA32F LUT, every miss of
the screen tracer (wavefront and megakernel, sun disk on primary misses),
the texel tracer and the probe baker reads the LUT as sample_sky_lut does
(scene.slang:469-518); the results equal the oracle's bit for bit (>= 99.9 %
of units exact, all within 1e-4 relative), and differ from the constant sky.
The sun transmittance helper reads a transmittance LUT at the reference's
view (scene.slang:997-1009)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _seeded_lut(h=200, w=200, seed=7):
    rng = np.random.default_rng(seed)
    yy, xx = np.meshgrid(np.linspace(0, 1, h), np.linspace(0, 1, w), indexing="ij")
    lut = np.zeros((h, w, 4), np.float32)
    lut[..., 0] = 0.1 + 0.4 * yy + 0.05 * rng.random((h, w))
    lut[..., 1] = 0.2 + 0.3 * np.sin(2 * np.pi * xx) ** 2
    lut[..., 2] = 0.4 + 0.3 * yy * (1 + np.cos(2 * np.pi * xx))
    lut[..., 3] = 1.0
    return lut


def _close(gpu, ref):
    exact = np.all(gpu == ref, axis=1)
    rel = np.max(np.abs(gpu - ref) / np.maximum(np.abs(ref), 1e-3), axis=1)
    assert exact.mean() >= 0.999, exact.mean()
    assert (rel <= 1e-4).mean() >= 0.999


@pytest.fixture(scope="module")
def sky_scene(device):
    import torch

    import nan_b200
    from nan_b200 import scenes
    from oracle.oracle import OracleScene

    node = scenes.terrain_boxes(seed=6, grid=65, boxes=30)
    scene = nan_b200.Scene(device, node)
    lut = torch.from_numpy(_seeded_lut()).cuda()
    scene.lighting = nan_b200.Lighting.sun_elevation(35.0, azimuth_deg=40.0, irradiance=3.0, sky=0.5,
                                                     sky_view_lut=lut)
    return node, scene, OracleScene(**scene.host)


@pytest.mark.parametrize("integrator", ["wavefront", "megakernel"])
def test_screen_misses_read_the_lut(sky_scene, device, integrator):
    import torch

    import nan_b200

    node, scene, orc = sky_scene
    scene.configure(integrator)
    w, h = 96, 64
    px = np.stack(np.meshgrid(np.arange(w), np.arange(h), indexing="xy"), -1).reshape(-1, 2)
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    for frame in (0, 3):
        node.camera.begin_frame(w, h)
        nan_b200.PathTracer(device, scene).execute(None, out, frame)
        ref, _ = orc.trace_screen(scene.lighting, node.camera, w, h, frame, 5, px)
        _close(out.cpu().numpy().reshape(-1, 4), ref)
    scene.configure("wavefront")
    device.check()


def test_texels_and_probes_read_the_lut(sky_scene, device):
    import torch

    import nan_b200
    from nan_b200.mesh_colors import MeshColorsLayout

    node, scene, orc = sky_scene
    layout = MeshColorsLayout.build(node, texels_per_unit=8.0, min_resolution=2, max_resolution=16)
    slots = torch.zeros((layout.total_payload_count, 4), dtype=torch.int32, device="cuda")
    nan_b200.TextureSpacePathTracer(device, scene, layout).execute(None, slots, 0, reset=True)
    host = np.zeros((layout.total_payload_count, 4), np.uint32)
    orc.trace_texels(scene.lighting, host, layout.face_array, layout.instance_array, layout.side_array,
                     layout.units(), 0, 1, 3, True)
    g = slots.cpu().numpy().view(np.uint32)
    assert np.mean(np.all(g == host, axis=1)) >= 0.999
    # the LUT changes the result
    const = nan_b200.Lighting.sun_elevation(35.0, azimuth_deg=40.0, irradiance=3.0, sky=0.5)
    host_c = np.zeros_like(host)
    orc.trace_texels(const, host_c, layout.face_array, layout.instance_array, layout.side_array, layout.units(),
                     0, 1, 3, True)
    assert np.mean(np.all(host_c == host, axis=1)) < 0.9

    from nan_b200 import scenes

    probes, pinst = scenes.surface_sites(node, 600, seed=4, radius=0.3)
    lay = type("L", (), {})()
    lay.probes = probes
    lay.nodes = np.zeros((1, 4), np.uint32)
    lay.instance_gpu_data = pinst
    lay.triangle_vertex_probes = np.zeros((1, 4), np.uint32)
    lay.total_probe_count = probes.shape[0]
    lay.instance_infos = list(range(pinst.shape[0]))
    geometry = nan_b200.SurfaceProbeGpuGeometry.create(device, lay)
    runtime = nan_b200.SurfaceProbeRuntimeBuffers.acquire(nan_b200.RenderData(device), probes.shape[0])
    baker = nan_b200.SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=8, max_bounces=3)
    baker.execute(None, runtime.field, runtime.attachments, 0, reset=True)
    n = probes.shape[0]
    values = np.zeros((n, 3), np.float32)
    counts = np.zeros(n, np.uint32)
    self_hits = np.zeros(n, np.uint32)
    radial = np.zeros((n, 16), np.uint32)
    orc.trace_probes(scene.lighting, values, counts, self_hits, radial, probes, pinst,
                     np.arange(n, dtype=np.uint32), 0, 8, 3, True)
    _close(runtime.field.values.cpu().numpy().view(np.float32).reshape(n, 3), values)
    device.check()


def test_sun_transmittance_from_lut():
    from nan_b200.scene import sun_transmittance_from_lut

    lut = np.zeros((64, 256, 4), np.float32)
    lut[..., 0] = np.linspace(0, 1, 256)[None, :]
    lut[..., 1] = 0.5
    lut[..., 2] = np.linspace(0, 1, 64)[:, None]
    t = sun_transmittance_from_lut(lut, (0.0, 1.0, 0.0))  # sun at the zenith: u = 1
    assert abs(t[0] - 1.0) < 1e-6 and abs(t[1] - 0.5) < 1e-6 and 0.0 <= t[2] <= 0.01
    t = sun_transmittance_from_lut(lut, (1.0, 0.0, 0.0))  # horizon: u = 1/2
    assert abs(t[0] - 0.5) < 0.01
