"""Point octree and probe-site layout (surface_probes.py:1348-1438,
2636-2950, 3016-3099 of the reference), pinned to vectors generated from the
reference's own builder and query (tests/golden/make_golden.py), plus the
layout invariants of test_surface_probes.py:916-972, and the kernels' own exp
and log2 against the C library."""

import math

import numpy as np
import pytest


@pytest.mark.parametrize("case", [0, 1, 2])
def test_octree_matches_reference_vectors(golden, case):
    from nan_b200.surface_probe_octree import build_point_octree

    leaf, depth = (int(x) for x in golden[f"octree{case}_params"])
    nodes, order, center, extent = build_point_octree(golden[f"octree{case}_positions"], leaf_capacity=leaf,
                                                      max_depth=depth)
    np.testing.assert_array_equal(nodes, golden[f"octree{case}_nodes"])
    np.testing.assert_array_equal(order, golden[f"octree{case}_order"])
    np.testing.assert_array_equal(np.array([*center, extent]), golden[f"octree{case}_root"])


def test_octree_query_matches_reference_vectors(golden):
    import types

    from nan_b200.surface_probe_octree import build_point_octree, query_probe_indices
    from nan_b200.surface_probe_resources import SURFACE_PROBE_DTYPE

    pos = golden["octree2_positions"]
    nodes, order, center, extent = build_point_octree(pos, leaf_capacity=8, max_depth=16)
    probes = np.zeros(pos.shape[0], dtype=SURFACE_PROBE_DTYPE)
    probes["position_radius"][:, :3] = pos[order]
    normals = np.zeros((pos.shape[0], 3), np.float32)
    normals[:3000, 1] = 1.0
    normals[3000:, 1] = -1.0
    probes["normal_side"][:, :3] = normals[order]
    info = types.SimpleNamespace(node_offset=0, root_center=center, root_extent=extent, kernel_radius=0.3)
    layout = types.SimpleNamespace(instance_infos=[info], nodes=nodes, probes=probes)
    q, radii, qn = golden["octree_query_positions"], golden["octree_query_radii"], golden["octree_query_normals"]
    found, off = golden["octree_query_found"], golden["octree_query_offsets"]
    for i in range(q.shape[0]):
        normal = None if not np.any(qn[i]) else qn[i]
        radius = None if radii[i] < 0 else float(radii[i])
        got = query_probe_indices(layout, 0, q[i], radius=radius, normal=normal)
        np.testing.assert_array_equal(got, found[off[i]:off[i + 1]])


def test_octree_rejects_empty_input():
    from nan_b200.surface_probe_octree import build_point_octree

    with pytest.raises(ValueError):
        build_point_octree(np.zeros((0, 3), np.float32))


def test_site_layout_ranges_and_queries():
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout

    node = scenes.cornell_box(16, 16)
    layout = SurfaceProbeSiteLayout.build(node, 900, seed=4)
    assert layout.probes.shape[0] == layout.total_probe_count
    assert sum(i.probe_count for i in layout.instance_infos) == layout.total_probe_count
    for k, info in enumerate(layout.instance_infos):
        node_end = info.node_offset + info.node_count
        probe_end = info.probe_offset + info.probe_count
        assert node_end <= layout.nodes.shape[0] and probe_end <= layout.probes.shape[0]
        inst = layout.probes["meta"][info.probe_offset:probe_end, 3] >> 8
        assert np.all(inst == k)
        for child_base, mask, start, count in layout.nodes[info.node_offset:node_end].astype(np.int64):
            if mask:
                assert info.node_offset <= child_base and child_base + bin(mask).count("1") <= node_end
            else:
                assert info.probe_offset <= start and start + count <= probe_end
        if info.probe_count == 0:
            continue
        found = layout.query_probe_indices(k, info.root_center, radius=info.root_extent * 4.0)
        np.testing.assert_array_equal(np.sort(found), np.arange(info.probe_offset, probe_end))
        first = layout.probes["position_radius"][info.probe_offset, :3]
        assert info.probe_offset in layout.query_probe_indices(k, first, radius=1e-7)
        gpu = layout.instance_gpu_data[k]
        assert tuple(gpu["offsets"]) == (info.node_offset, info.node_count, info.probe_offset, info.probe_count)
        assert gpu["params"][0] == np.float32(info.kernel_radius) and gpu["params"][2] == np.float32(
            max(info.kernel_radius * 0.25, 1e-6))
        np.testing.assert_array_equal(layout.probes["position_radius"][info.probe_offset:probe_end, 3],
                                      np.float32(info.kernel_radius))
    assert np.all(layout.triangle_vertex_probes[:, 3] == 0)


def test_own_exp_and_log2_within_two_ulp():
    from oracle.oracle import own_exp, own_log2

    rng = np.random.default_rng(5)
    xs = np.concatenate([rng.uniform(-87.0, 88.0, 3000), rng.uniform(-8.0, 0.0, 3000), [0.0, -0.0, 1.0, -1.0]])
    for x in xs.astype(np.float32):
        want = np.float32(math.exp(float(x)))
        got = np.float32(own_exp(float(x)))
        assert abs(int(got.view(np.int32)) - int(want.view(np.int32))) <= 2, (x, got, want)
    ys = np.concatenate([np.exp2(rng.uniform(-140.0, 120.0, 3000)), rng.uniform(1e-6, 10.0, 3000), [1.0, 2.0, 10.0]])
    for y in ys.astype(np.float32):
        if y == 0:
            continue
        want = math.log2(float(y))
        got = own_log2(float(y))
        assert abs(got - want) <= 2.5 * abs(float(np.spacing(np.float32(want)))) + 1e-7, (y, got, want)
    assert own_exp(-100.0) == 0.0 and math.isinf(own_exp(100.0)) and own_log2(8.0) == 3.0


@pytest.mark.parametrize("leaf,depth", [(8, 16), (1, 16), (3, 5)])
def test_octree_matches_reference_cpp_builder(leaf, depth):
    """The reference's default (C++) builder, compiled from its sources,
    gives the same nodes, order and root as the host builder."""
    from nan_b200.surface_probe_octree import build_point_octree
    from oracle import ref_sampler

    if not ref_sampler.available():
        pytest.skip("reference sampler library not built")
    rng = np.random.default_rng(leaf * 10 + depth)
    p = rng.normal(size=(3000, 3)).astype(np.float32)
    p[:600] = p[0]
    p[600:1000, 1] = 0.0
    ref = ref_sampler.build_point_octree(p, leaf_capacity=leaf, max_depth=depth)
    mine = build_point_octree(p, leaf_capacity=leaf, max_depth=depth)
    np.testing.assert_array_equal(mine[0], ref[0])
    np.testing.assert_array_equal(mine[1], ref[1])
    assert mine[2] == ref[2] and mine[3] == ref[3]
