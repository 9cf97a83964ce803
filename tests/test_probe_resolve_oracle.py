"""Surface-probe resolve on the oracle (CPU): a constant irradiance field on
a plane reconstructs to that constant (albedo / pi * E on every hit pixel),
every hit pixel gathers probes, empty radial moments leave the visibility
prior neutral, the fallback merge keeps at most 32 probes, and an
out-of-range octree index is reported."""

import math

import numpy as np
import pytest


def _plane_scene(w=24, h=16):
    from nan_b200 import scenes
    from nan_b200.scene_node import Material, Mesh, SceneNode

    v = np.zeros((4, 8), np.float32)
    v[:, :3] = [(-4, 0, -4), (4, 0, -4), (4, 0, 4), (-4, 0, 4)]
    v[:, 4] = 1.0
    node = SceneNode(name="plane")
    mesh = node.add_mesh(Mesh(v, np.array([[0, 2, 1], [0, 3, 2]], np.uint32)))
    node.add_instance(mesh, node.add_material(Material(base_color=(0.5, 0.25, 1.0))),
                      node.add_transform(np.eye(4, dtype=np.float32)))
    node.camera = scenes._camera((0.0, 3.0, 3.0), (0.0, 0.0, 0.0), 50.0, w, h)
    node.camera.begin_frame(w, h)
    return node


def _resolve(node, layout, values, counts, radial=None, **kw):
    from nan_b200.scene import Lighting
    from oracle.oracle import OracleScene

    orc = OracleScene(**node.pack())
    w, h = node.camera.width, node.camera.height
    px = np.stack(np.meshgrid(np.arange(w), np.arange(h), indexing="xy"), -1).reshape(-1, 2)
    n = layout.total_probe_count
    light = Lighting(sun_intensity=0.0, sky_radiance=(0.0, 0.0, 0.0), sun_disk=False)
    radial = np.zeros((n, 16), np.uint32) if radial is None else radial
    return orc.resolve_probes(light, node.camera, w, h, px, layout, values, counts, np.zeros(n, np.uint32), radial,
                              **kw)


def test_constant_field_reconstructs_to_the_constant():
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout

    node = _plane_scene()
    layout = SurfaceProbeSiteLayout.build(node, 400, seed=2)
    n = layout.total_probe_count
    e = np.array([2.0, 3.0, 0.5], np.float32)
    values = np.tile(e, (n, 1))
    counts = np.full(n, 5, np.uint32)
    out = _resolve(node, layout, values, counts)
    hit = np.any(out[:, :3] != 0.0, axis=1)
    assert hit.mean() > 0.5
    want = np.array([0.5, 0.25, 1.0], np.float32) * np.float32(1.0 / math.pi) * e
    np.testing.assert_allclose(out[hit, :3], np.broadcast_to(want, (int(hit.sum()), 3)), rtol=1e-6)
    counts_view = _resolve(node, layout, values, counts, debug_view=1)
    magenta = np.all(counts_view[hit, :3] == np.float32([1, 0, 1]), axis=1)
    assert not magenta.any()
    # without samples the probes carry no weight: the strongest probe's value is used
    zero = _resolve(node, layout, values, np.zeros(n, np.uint32))
    np.testing.assert_allclose(zero[hit, :3], out[hit, :3], rtol=1e-6)


def test_empty_moments_leave_visibility_neutral_and_gather_is_capped():
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout

    node = _plane_scene()
    layout = SurfaceProbeSiteLayout.build(node, 3000, seed=3)
    n = layout.total_probe_count
    rng = np.random.default_rng(1)
    values = rng.uniform(0.0, 4.0, (n, 3)).astype(np.float32)
    counts = np.full(n, 40, np.uint32)
    a = _resolve(node, layout, values, counts, use_radial_visibility=True)
    b = _resolve(node, layout, values, counts, use_radial_visibility=False)
    np.testing.assert_array_equal(a, b)
    # about 20 sites fall inside the kernel radius (2.5 x the mean spacing): the
    # gather-count view shows 8..23 (red channel 0) on most hit pixels
    hit = np.any(a[:, :3] != 0.0, axis=1)
    view = _resolve(node, layout, values, counts, debug_view=1)
    assert np.mean(view[hit, 0] == 0.0) > 0.8
    # asking for 32 starts the 2R fallback, which fills the gather to its cap of 32 (white)
    capped = _resolve(node, layout, values, counts, debug_view=1, min_gather_count=32)
    white = np.all(capped[hit, :3] == np.float32([1, 1, 1]), axis=1)
    assert white.mean() > 0.8


def test_out_of_range_node_is_reported():
    import dataclasses

    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout

    node = _plane_scene()
    layout = SurfaceProbeSiteLayout.build(node, 200, seed=2)
    bad_nodes = layout.nodes.copy()
    branch = np.flatnonzero(bad_nodes[:, 1] != 0)
    bad_nodes[branch[0], 0] = bad_nodes.shape[0] + 5
    bad = dataclasses.replace(layout, nodes=bad_nodes)
    n = layout.total_probe_count
    with pytest.raises(RuntimeError):
        _resolve(node, bad, np.ones((n, 3), np.float32), np.ones(n, np.uint32))
