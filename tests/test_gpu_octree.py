"""Point octrees on the GPU (nan_build_point_octrees) against the
reference's builder: the golden vectors made by its own Python builder
(nodes, order, root), its C++ builder compiled from its sources, and the
host restatement (build_point_octree) on many
sets in one call, with clustered and coincident points and depth limits; a
site layout packed with the GPU octrees equals the host-packed one."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [0, 1, 2])
def test_gpu_octree_matches_reference_vectors(golden, device, case):
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    leaf, depth = (int(x) for x in golden[f"octree{case}_params"])
    (nodes, order, center, extent), = SurfaceProbeSampler(device).build_point_octrees(
        [golden[f"octree{case}_positions"]], leaf_capacity=leaf, max_depth=depth)
    np.testing.assert_array_equal(nodes, golden[f"octree{case}_nodes"])
    np.testing.assert_array_equal(order, golden[f"octree{case}_order"])
    np.testing.assert_array_equal(np.array([*center, extent]), golden[f"octree{case}_root"])


@pytest.mark.parametrize("leaf,depth", [(8, 16), (1, 16), (3, 5), (16, 2)])
def test_gpu_octrees_match_host_builder(device, leaf, depth):
    from nan_b200.surface_probe_octree import build_point_octree
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    rng = np.random.default_rng(leaf * 100 + depth)
    sets = []
    for k in range(23):
        n = int(rng.integers(0, 3000)) if k % 7 else int(rng.integers(1, 5))
        p = rng.normal(size=(n, 3)).astype(np.float32) * rng.uniform(0.01, 50.0)
        if n > 10:
            p[: n // 5] = p[0]  # coincident points
            p[n // 5: n // 3, 1] = 0.0  # a flat cluster
        sets.append(p + rng.uniform(-100, 100, 3).astype(np.float32))
    sets.append(np.zeros((0, 3), np.float32))
    trees = SurfaceProbeSampler(device).build_point_octrees(sets, leaf_capacity=leaf, max_depth=depth)
    for p, tree in zip(sets, trees):
        if p.shape[0] == 0:
            assert tree is None
            continue
        nodes, order, center, extent = build_point_octree(p, leaf_capacity=leaf, max_depth=depth)
        np.testing.assert_array_equal(tree[0], nodes)
        np.testing.assert_array_equal(tree[1], order)
        assert tree[2] == center and tree[3] == extent
    device.check()


def test_gpu_octrees_match_reference_cpp_builder(device):
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler
    from oracle import ref_sampler

    if not ref_sampler.available():
        pytest.skip("reference sampler library not built")
    rng = np.random.default_rng(17)
    sets = [rng.normal(size=(int(n), 3)).astype(np.float32) * 3.0 for n in rng.integers(1, 20000, 6)]
    for leaf, depth in ((8, 16), (2, 9)):
        trees = SurfaceProbeSampler(device).build_point_octrees(sets, leaf_capacity=leaf, max_depth=depth)
        for p, tree in zip(sets, trees):
            ref = ref_sampler.build_point_octree(p, leaf_capacity=leaf, max_depth=depth)
            np.testing.assert_array_equal(tree[0], ref[0])
            np.testing.assert_array_equal(tree[1], ref[1])
            assert tree[2] == ref[2] and tree[3] == ref[3]
    device.check()


def test_layout_packed_on_gpu_equals_host(device):
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    node = scenes.terrain_boxes(seed=3, grid=97, boxes=30)
    probes, _ = scenes.surface_sites(node, 5000, seed=2)
    host = SurfaceProbeSiteLayout.from_sites(node, probes)
    gpu = SurfaceProbeSiteLayout.from_sites(node, probes, sampler=SurfaceProbeSampler(device))
    np.testing.assert_array_equal(gpu.probes, host.probes)
    np.testing.assert_array_equal(gpu.nodes, host.nodes)
    np.testing.assert_array_equal(gpu.instance_gpu_data, host.instance_gpu_data)
    device.check()
