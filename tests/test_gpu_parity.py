"""CUDA path vs the CPU oracle on the same seeded inputs (GPU required).

The oracle's float mode follows the same operation order as the kernels, so
the expected agreement is bit-exact; the FP64 brute force bounds the
intersection itself (>= 99.99 % identical hit ids, t within 1e-6 relative).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _build(device, node, bvh_builder="sah"):
    import nan_b200

    scene = nan_b200.Scene(device, node, bvh_builder=bvh_builder)
    from oracle.oracle import OracleScene

    return scene, OracleScene(**scene.host)


def _random_rays(world_tris, n, seed, inside=True):
    rng = np.random.default_rng(seed)
    pts = world_tris.reshape(-1, 3)
    lo, hi = pts.min(0), pts.max(0)
    ext = hi - lo
    o = rng.uniform(lo - 0.1 * ext, hi + 0.1 * ext, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 0.0
    rays[:, 4:7] = d
    rays[:, 7] = 1e30
    # some rays start exactly on a surface point toward random directions
    k = n // 4
    tri = world_tris[rng.integers(0, world_tris.shape[0], k)].reshape(k, 3, 3).astype(np.float64)
    b = rng.dirichlet([1, 1, 1], size=k)
    rays[:k, 0:3] = np.einsum("kj,kjc->kc", b, tri).astype(np.float32)
    rays[:k, 3] = 1e-4
    return rays


@pytest.fixture(scope="module")
def cornell(device):
    from nan_b200 import scenes

    return _build(device, scenes.cornell_box(64, 64))


@pytest.fixture(scope="module")
def terrain(device):
    from nan_b200 import scenes

    return _build(device, scenes.terrain_boxes(seed=1, grid=129, boxes=120))


@pytest.fixture(scope="module")
def terrain_lbvh(device):
    from nan_b200 import scenes

    return _build(device, scenes.terrain_boxes(seed=1, grid=129, boxes=120), bvh_builder="lbvh")


@pytest.fixture(scope="module")
def terrain_ploc(device):
    from nan_b200 import scenes

    return _build(device, scenes.terrain_boxes(seed=1, grid=129, boxes=120), bvh_builder="ploc")


@pytest.mark.parametrize("which", ["cornell", "terrain", "terrain_lbvh", "terrain_ploc"])
def test_bvh_world_triangles_match_oracle(which, request):
    scene, orc = request.getfixturevalue(which)
    np.testing.assert_array_equal(scene.world_triangles().cpu().numpy(), orc.world_triangles())
    info = scene.info()
    assert info["triangle_count"] == orc.triangle_count
    assert info["max_depth"] <= 96
    if scene.bvh_builder == "ploc":  # SAH quality close to the binned-SAH reference
        assert info["sah_cost"] <= 1.25 * orc.bvh_stats()["sah_cost"], (info["sah_cost"], orc.bvh_stats())
    if scene.bvh_builder == "sah":
        assert info["sah_cost"] <= 1.05 * orc.bvh_stats()["sah_cost"], (info["sah_cost"], orc.bvh_stats())


@pytest.mark.parametrize("width", [2, 8])
@pytest.mark.parametrize("which", ["cornell", "terrain", "terrain_lbvh", "terrain_ploc"])
def test_closest_hit_bit_exact_vs_oracle(which, width, request):
    import torch

    scene, orc = request.getfixturevalue(which)
    scene.configure(bvh_width=width)
    rays = _random_rays(orc.world_triangles(), 20000, seed=7)
    ids, tb = scene.intersect(torch.from_numpy(rays).cuda())
    ids = ids.cpu().numpy().view(np.uint32)
    tb = tb.cpu().numpy()
    o_ids, o_tb, _ = orc.intersect(rays, mode=0)
    np.testing.assert_array_equal(ids, o_ids)
    valid = ids[:, 0] == 1
    np.testing.assert_array_equal(tb[valid], o_tb[valid])
    assert valid.mean() > 0.3
    scene.configure()


@pytest.mark.parametrize("which", ["cornell", "terrain"])
def test_closest_hit_vs_fp64_bruteforce(which, request):
    """FP32 watertight hits vs an FP64 brute force on rays from random origins:
    >= 99.99 % identical ids, every disagreement a t-tie within 1e-6 relative."""
    import torch

    scene, orc = request.getfixturevalue(which)
    rays = _random_rays(orc.world_triangles(), 20000, seed=11)
    rays = rays[rays.shape[0] // 4:]  # drop the rays that start on a surface
    ids, tb = scene.intersect(torch.from_numpy(rays).cuda())
    ids = ids.cpu().numpy().view(np.uint32)
    tb = tb.cpu().numpy()
    d_ids, d_tb, _ = orc.intersect(rays, mode=2)
    same = (ids[:, 0] == d_ids[:, 0]) & ((ids[:, 0] == 0) | (ids[:, 3] == d_ids[:, 3]))
    both = (ids[:, 0] == 1) & (d_ids[:, 0] == 1) & ~same
    tie = np.abs(tb[both, 0] - d_tb[both, 0]) <= 1e-6 * np.maximum(np.abs(d_tb[both, 0]), 1e-3)
    ok = same.copy()
    ok[np.where(both)[0][tie]] = True
    assert ok.mean() >= 0.9999, (ok.mean(), np.where(~ok)[0][:10], tb[~ok, 0], d_tb[~ok, 0])
    hit = (ids[:, 0] == 1) & same
    rel_t = np.abs(tb[hit, 0] - d_tb[hit, 0]) / np.maximum(np.abs(d_tb[hit, 0]), 1e-3)
    assert np.median(rel_t) <= 1e-6 and np.quantile(rel_t, 0.99) <= 1e-5, np.quantile(rel_t, [0.5, 0.99, 1])


@pytest.mark.parametrize("width", [2, 8])
@pytest.mark.parametrize("which", ["cornell", "terrain", "terrain_lbvh", "terrain_ploc"])
def test_any_hit_bit_exact_vs_oracle(which, width, request):
    import torch

    scene, orc = request.getfixturevalue(which)
    scene.configure(bvh_width=width)
    rays = _random_rays(orc.world_triangles(), 20000, seed=9)
    rays[:, 7] = np.random.default_rng(1).uniform(0.01, 3.0, rays.shape[0]).astype(np.float32)
    vis = scene.occluded(torch.from_numpy(rays).cuda()).cpu().numpy()
    o_vis, _ = orc.visibility(rays, mode=0)
    np.testing.assert_array_equal(vis, o_vis)
    assert 0.05 < vis.mean() < 0.95
    scene.configure()


@pytest.mark.parametrize("which", ["cornell", "terrain"])
def test_screen_path_tracer_matches_oracle(which, request, device):
    import torch

    import nan_b200

    scene, orc = request.getfixturevalue(which)
    cam = scene.camera
    w = h = 64
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    tracer = nan_b200.PathTracer(device, scene)
    for frame in (0, 5):
        cam.begin_frame(w, h)
        tracer.execute(None, out, frame)
        gpu = out.cpu().numpy().reshape(-1, 4)
        px = np.stack(np.meshgrid(np.arange(w), np.arange(h), indexing="xy"), -1).reshape(-1, 2)
        ref, _ = orc.trace_screen(scene.lighting, cam, w, h, frame, 5, px)
        exact = np.all(gpu == ref, axis=1)
        rel = np.max(np.abs(gpu - ref) / np.maximum(np.abs(ref), 1e-3), axis=1)
        assert exact.mean() >= 0.999, exact.mean()
        assert (rel <= 1e-4).mean() >= 0.999
    device.check()


def _layout_and_buffers(device, scene):
    import torch

    from nan_b200.mesh_colors import MeshColorsLayout

    layout = MeshColorsLayout.build(scene.scene_node, texels_per_unit=16.0, min_resolution=4, max_resolution=64)
    slots = torch.zeros((layout.total_payload_count, 4), dtype=torch.int32, device="cuda")
    return layout, slots


@pytest.mark.parametrize("integrator", ["wavefront", "megakernel"])
@pytest.mark.parametrize("which", ["cornell", "terrain"])
def test_texel_tracer_matches_oracle(which, integrator, request, device):
    import nan_b200

    scene, orc = request.getfixturevalue(which)
    scene.configure(integrator)
    if which == "terrain":
        scene.lighting = nan_b200.Lighting.sun_elevation(45.0, azimuth_deg=30.0, irradiance=3.0, sky=0.5)
    layout, slots = _layout_and_buffers(device, scene)
    tracer = nan_b200.TextureSpacePathTracer(device, scene, layout, samples_per_texel=1, max_bounces=3)
    rng = np.random.default_rng(5)
    units = layout.units()
    pick = units[rng.choice(units.shape[0], size=min(3000, units.shape[0]), replace=False)]
    host = np.zeros((layout.total_payload_count, 4), np.uint32)
    for it in range(3):
        tracer.execute(None, slots, it, reset=(it == 0))
        orc.trace_texels(scene.lighting, host, layout.face_array, layout.instance_array, layout.side_array,
                         pick, it, 1, 3, it == 0)
    gpu = slots.cpu().numpy().view(np.uint32)
    # compare the slots the picked units wrote (front, and back if double sided)
    inst = layout.instance_array[pick[:, 0]]
    front = inst[:, 2] + pick[:, 1]
    idx = [front]
    side = layout.side_array[pick[:, 0]]
    ds = (side[:, 1] & 1) == 1
    idx.append(side[ds, 0] + pick[ds, 1])
    idx = np.concatenate(idx)
    g = gpu[idx]
    o = host[idx]
    assert np.all(g[:, 3] == 3) and np.all(o[:, 3] == 3)
    exact = np.all(g == o, axis=1)
    gv, ov = g[:, :3].view(np.float32), o[:, :3].view(np.float32)
    rel = np.max(np.abs(gv - ov) / np.maximum(np.abs(ov), 1e-3), axis=1)
    assert exact.mean() >= 0.999, exact.mean()
    assert (rel <= 1e-4).mean() >= 0.999
    device.check()
    scene.configure("wavefront")


@pytest.mark.parametrize("spt,chunk", [(1, 0), (2, 5000), (1, 777)])
def test_texel_wavefront_equals_megakernel(terrain, device, spt, chunk):
    """Every slot of the full layout, several iterations, chunked wavefronts."""
    import torch

    import nan_b200

    scene, _ = terrain
    scene.lighting = nan_b200.Lighting.sun_elevation(45.0, azimuth_deg=30.0, irradiance=3.0, sky=0.5)
    layout, slots_a = _layout_and_buffers(device, scene)
    slots_b = torch.zeros_like(slots_a)
    tracer = nan_b200.TextureSpacePathTracer(device, scene, layout, samples_per_texel=spt, max_bounces=3)
    for it in range(2):
        scene.configure("megakernel")
        tracer.execute(None, slots_a, it, reset=(it == 0))
        scene.configure("wavefront", max_paths_in_flight=chunk)
        tracer.execute(None, slots_b, it, reset=(it == 0))
    scene.configure("wavefront")
    torch.testing.assert_close(slots_b, slots_a, rtol=0, atol=0)
    device.check()


def test_texel_wavefront_two_sided(cornell, device):
    """Cornell walls are double sided: back slots run after the front path."""
    import torch

    import nan_b200

    scene, _ = cornell
    layout, slots_a = _layout_and_buffers(device, scene)
    assert (layout.side_array[:, 1] & 1).any()
    slots_b = torch.zeros_like(slots_a)
    tracer = nan_b200.TextureSpacePathTracer(device, scene, layout, samples_per_texel=3, max_bounces=4)
    for it in range(2):
        scene.configure("megakernel")
        tracer.execute(None, slots_a, it, reset=(it == 0))
        scene.configure("wavefront")
        tracer.execute(None, slots_b, it, reset=(it == 0))
    torch.testing.assert_close(slots_b, slots_a, rtol=0, atol=0)
    device.check()


def test_screen_wavefront_equals_megakernel(cornell, terrain, device):
    import torch

    import nan_b200

    for scene, _ in (cornell, terrain):
        cam = scene.camera
        w, h = 96, 64
        a = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
        b = torch.zeros_like(a)
        tracer = nan_b200.PathTracer(device, scene)
        for frame in (0, 7):
            cam.begin_frame(w, h)
            scene.configure("megakernel")
            tracer.execute(None, a, frame)
            scene.configure("wavefront", max_paths_in_flight=1000)
            tracer.execute(None, b, frame)
            torch.testing.assert_close(b, a, rtol=0, atol=0)
        scene.configure("wavefront")
    device.check()


def _probe_setup(device, scene, count, spp):
    import nan_b200
    from nan_b200 import scenes

    probes, pinst = scenes.surface_sites(scene.scene_node, count, seed=3, radius=0.3)
    layout = type("L", (), {})()
    layout.probes = probes
    layout.nodes = np.zeros((1, 4), np.uint32)
    layout.instance_gpu_data = pinst
    layout.triangle_vertex_probes = np.zeros((1, 4), np.uint32)
    layout.total_probe_count = probes.shape[0]
    layout.instance_infos = list(range(pinst.shape[0]))
    geometry = nan_b200.SurfaceProbeGpuGeometry.create(device, layout)
    baker = nan_b200.SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=spp,
                                                        max_bounces=3)
    return probes, pinst, geometry, baker


def test_probe_wavefront_equals_megakernel(terrain, device):
    import torch

    import nan_b200

    scene, _ = terrain
    probes, pinst, geometry, baker = _probe_setup(device, scene, 3000, 12)
    runs = []
    for integrator in ("megakernel", "wavefront"):
        scene.configure(integrator, max_paths_in_flight=1111 if integrator == "wavefront" else 0)
        rd = nan_b200.RenderData(device)
        runtime = nan_b200.SurfaceProbeRuntimeBuffers.acquire(rd, probes.shape[0])
        for it in range(3):
            baker.execute(None, runtime.field, runtime.attachments, it, reset=(it == 0))
        runs.append([runtime.field.values.clone(), runtime.field.sample_counts.clone(),
                     runtime.attachments.self_hit_counts.clone(), runtime.attachments.radial_moments.clone()])
    scene.configure("wavefront")
    for x, y in zip(*runs):
        torch.testing.assert_close(y, x, rtol=0, atol=0)
    device.check()


def test_probe_baker_matches_oracle(terrain, device):
    import torch

    import nan_b200
    from nan_b200 import scenes

    scene, orc = terrain
    probes, pinst = scenes.surface_sites(scene.scene_node, 2000, seed=3, radius=0.3)
    layout = type("L", (), {})()
    layout.probes = probes
    layout.nodes = np.zeros((1, 4), np.uint32)
    layout.instance_gpu_data = pinst
    layout.triangle_vertex_probes = np.zeros((1, 4), np.uint32)
    layout.total_probe_count = probes.shape[0]
    layout.instance_infos = list(range(pinst.shape[0]))
    geometry = nan_b200.SurfaceProbeGpuGeometry.create(device, layout)
    rd = nan_b200.RenderData(device)
    runtime = nan_b200.SurfaceProbeRuntimeBuffers.acquire(rd, probes.shape[0])
    baker = nan_b200.SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=8, max_bounces=3)
    n = probes.shape[0]
    values = np.zeros((n, 3), np.float32)
    counts = np.zeros(n, np.uint32)
    self_hits = np.zeros(n, np.uint32)
    radial = np.zeros((n, 16), np.uint32)
    units = np.arange(n, dtype=np.uint32)
    for it in range(3):
        baker.execute(None, runtime.field, runtime.attachments, it, reset=(it == 0))
        orc.trace_probes(scene.lighting, values, counts, self_hits, radial, probes, pinst, units, it, 8, 3, it == 0)
    g_values = runtime.field.values.cpu().numpy().view(np.float32).reshape(n, 3)
    g_counts = runtime.field.sample_counts.cpu().numpy().view(np.uint32)
    g_self = runtime.attachments.self_hit_counts.cpu().numpy().view(np.uint32)
    g_radial = runtime.attachments.radial_moments.cpu().numpy().view(np.uint32).reshape(n, 16)
    np.testing.assert_array_equal(g_counts, counts)
    exact = np.all(g_values == values, axis=1) & (g_self == self_hits) & np.all(g_radial == radial, axis=1)
    assert exact.mean() >= 0.999, exact.mean()
    device.check()


def test_accumulator_matches_numpy(device):
    import torch

    import nan_b200

    rd = nan_b200.RenderData(device)
    acc = nan_b200.Accumulator(device)
    rng = np.random.default_rng(2)
    h, w = 37, 53
    hist = np.zeros((h, w, 4), np.float32)
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    for k in range(4):
        frame = rng.uniform(0, 10, (h, w, 4)).astype(np.float32)
        acc.execute(None, rd, torch.from_numpy(frame).cuda(), out, reset=(k == 0))
        if k == 0:
            hist[:] = 0
        hist[..., :3] += frame[..., :3]
        hist[..., 3] += np.float32(1.0)
        expect = np.concatenate([hist[..., :3] / hist[..., 3:4], np.ones((h, w, 1), np.float32)], -1)
        np.testing.assert_array_equal(out.cpu().numpy(), expect)


def test_rgb9e5_pack_bit_exact_vs_reference(golden, device):
    import torch

    import nan_b200

    vals = golden["rgb9e5_values"]
    slots = np.zeros((vals.shape[0], 4), np.float32)
    slots[:, :3] = vals
    out = torch.zeros((vals.shape[0],), dtype=torch.int32, device="cuda")
    nan_b200.MeshColorsRGB9E5Packer(device).execute(None, torch.from_numpy(slots).cuda(), out, vals.shape[0])
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), golden["rgb9e5_packed"])
