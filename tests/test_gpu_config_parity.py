"""Parity on the workloads the benchmarks time, as generated.

The other parity tests run small scenes (about 33k triangles) and small
images. These run each benchmarked configuration with its own scene,
resolution, layout and ray length, trace it on the GPU in full, and compare
a seeded sample of its units with the oracle in float mode (the kernels'
operation order, so bit-exact agreement is expected; the bar is >= 99.9 % of
units bit for bit and >= 99.9 % within 1e-4 relative):

* config 1: the 36-triangle Cornell box at 256x256, frames 0 and 15, 4 path
  vertices (3 bounces), BSDF-only and with area-light NEE + MIS;
* config 2: the 200,688-triangle terrain + boxes, Mesh Colors layout at 16
  texels/unit, resolution 4-64 (12.6 M texels), two iterations;
* config 3: the 998,408-triangle terrain + 2000 boxes at 1920x1080, 5 path
  vertices, frames 0 and 1;
* config 5: the 4.16 M-triangle city with ray length 5000 (its diagonal
  exceeds the reference's 1000) at 3840x2160, 5 path vertices, and its
  12.6 M-texel Mesh Colors pass.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pixels(w, h, n, seed):
    rng = np.random.default_rng(seed)
    flat = rng.choice(w * h, size=n, replace=False)
    return np.stack([flat % w, flat // w], axis=1).astype(np.int64)


def _assert_close(gpu, ref):
    exact = np.all(gpu == ref, axis=1)
    rel = np.max(np.abs(gpu - ref) / np.maximum(np.abs(ref), 1e-3), axis=1)
    assert exact.mean() >= 0.999, exact.mean()
    assert (rel <= 1e-4).mean() >= 0.999, (rel <= 1e-4).mean()
    return exact.mean()


def _screen(device, scene, orc, w, h, frames, max_vertices, samples, seed):
    import torch

    import nan_b200

    cam = scene.camera
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    tracer = nan_b200.PathTracer(device, scene, max_vertices=max_vertices)
    for frame in frames:
        cam.begin_frame(w, h)
        tracer.execute(None, out, frame)
        px = _pixels(w, h, samples, seed + frame)
        gpu = out[torch.from_numpy(px[:, 1]).cuda(), torch.from_numpy(px[:, 0]).cuda()].cpu().numpy()
        ref, _ = orc.trace_screen(scene.lighting, cam, w, h, frame, max_vertices, px.astype(np.uint32))
        _assert_close(gpu, ref)
    device.check()


def _texels(device, scene, orc, layout, iterations, samples, seed):
    import torch

    import nan_b200

    slots = torch.zeros((layout.total_payload_count, 4), dtype=torch.int32, device="cuda")
    tracer = nan_b200.TextureSpacePathTracer(device, scene, layout, samples_per_texel=1, max_bounces=3)
    units = layout.units()
    rng = np.random.default_rng(seed)
    pick = units[rng.choice(units.shape[0], size=min(samples, units.shape[0]), replace=False)]
    host = np.zeros((layout.total_payload_count, 4), np.uint32)
    for it in range(iterations):
        tracer.execute(None, slots, it, reset=(it == 0))
        orc.trace_texels(scene.lighting, host, layout.face_array, layout.instance_array, layout.side_array,
                         pick, it, 1, 3, it == 0)
    inst = layout.instance_array[pick[:, 0]]
    idx = [inst[:, 2] + pick[:, 1]]
    side = layout.side_array[pick[:, 0]]
    ds = (side[:, 1] & 1) == 1
    idx.append(side[ds, 0] + pick[ds, 1])
    idx = np.concatenate(idx)
    g = slots.cpu().numpy().view(np.uint32)[idx]
    o = host[idx]
    assert np.all(g[:, 3] == iterations) and np.all(o[:, 3] == iterations)
    assert np.mean(np.all(g == o, axis=1)) >= 0.999
    _assert_close(g[:, :3].view(np.float32), o[:, :3].view(np.float32))
    device.check()


@pytest.mark.parametrize("area", [False, True])
def test_config1_cornell_256(device, area):
    import nan_b200
    from nan_b200 import scenes
    from oracle.oracle import OracleScene

    node = scenes.cornell_box(256, 256)
    scene = nan_b200.Scene(device, node)
    orc = OracleScene(**scene.host)
    if area:
        scene.enable_area_lights()
        table, power = scene.area_light_table()
        orc.set_area_lights(table, power)
    scene.lighting.area_nee = area
    _screen(device, scene, orc, 256, 256, (0, 15), 4, 4096, seed=11)


def test_config2_texels_200k(device):
    import nan_b200
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout
    from oracle.oracle import OracleScene

    node = scenes.terrain_boxes(seed=1, grid=313, boxes=500)
    scene = nan_b200.Scene(device, node)
    assert scene.triangle_count == 200_688
    layout = MeshColorsLayout.build(node, texels_per_unit=16.0, min_resolution=4, max_resolution=64)
    assert layout.total_surface_texels > 12_000_000
    _texels(device, scene, OracleScene(**scene.host), layout, 2, 3000, seed=21)


def test_config3_screen_998k(device):
    import nan_b200
    from nan_b200 import scenes
    from oracle.oracle import OracleScene

    node = scenes.terrain_boxes(seed=1, grid=699, boxes=2000)
    scene = nan_b200.Scene(device, node)
    assert scene.triangle_count == 998_408
    _screen(device, scene, OracleScene(**scene.host), 1920, 1080, (0, 1), 5, 3000, seed=31)


@pytest.fixture(scope="module")
def city(device):
    import nan_b200
    from nan_b200 import scenes
    from oracle.oracle import OracleScene

    node = scenes.city(width=3840, height=2160)
    node.lighting.ray_t_max = 5000.0
    scene = nan_b200.Scene(device, node)
    assert scene.triangle_count == 4_160_000
    return node, scene, OracleScene(**scene.host)


def test_config5_city_screen(device, city):
    _, scene, orc = city
    _screen(device, scene, orc, 3840, 2160, (0, 3), 5, 2000, seed=41)


def test_config5_city_texels(device, city):
    from nan_b200.mesh_colors import MeshColorsLayout

    node, scene, orc = city
    layout = MeshColorsLayout.build(node, texels_per_unit=0.1, min_resolution=1, max_resolution=64)
    _texels(device, scene, orc, layout, 1, 2000, seed=51)
