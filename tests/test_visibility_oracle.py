"""The PMR visibility caster's CPU restatement, pinned to the reference.

* The library's host-side ray table (nan_visibility_ray_table, the GPU
  kernel's input) equals the oracle's restatement of make_ray_projections
  (vertex_baker/cpp/tinybvh_visibility.cpp:52-101) bit for bit.
* The oracle's caster loop -- the same rays, the oracle's watertight any-hit
  (bit-exact with the GPU's), the caster's SH summation order -- is compared
  with the reference's own caster, compiled from its sources
  (vbake_pmr_visibility_sh_tinybvh, scalar BVH layout with its watertight
  triangle test), on the same world triangles and samples, with the
  reference benchmark's comparison (benchmark_tinybvh_visibility.py:45-61).
"""

import ctypes

import numpy as np
import pytest

from oracle import visibility as ov


def _sites(node, count, seed):
    from nan_b200 import scenes

    probes, _ = scenes.surface_sites(node, count, seed=seed, double_sided_backs=False)
    return (np.ascontiguousarray(probes["position_radius"][:, :3]),
            np.ascontiguousarray(probes["normal_side"][:, :3]))


@pytest.mark.parametrize("rays", [1, 7, 64, 100, 512, 1024])
def test_library_ray_table_equals_oracle(rays):
    from nan_b200 import visibility

    a = visibility.visibility_ray_table(rays)
    b = ov.ray_table(rays)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))


def test_ray_table_rejects_bad_counts():
    from nan_b200 import visibility

    for bad in (0, 1025):
        with pytest.raises(ValueError):
            visibility.visibility_ray_table(bad)


def test_sh_sum_follows_the_caster_batches():
    table = ov.ray_table(130)
    masks = np.zeros((2, 130), bool)
    masks[0] = True
    sh = ov.sum_sh16(masks, table)
    expect = np.float32(0)
    for b in range(0, 130, 64):
        batch = np.float32(0)
        for r in range(b, min(b + 64, 130)):
            batch = np.float32(batch + table[r, 4])
        expect = np.float32(expect + batch)
    assert sh[0, 0] == expect
    assert np.all(sh[1] == 0)


@pytest.mark.parametrize("max_distance", [1000.0, 0.5])
def test_oracle_caster_agrees_with_reference_caster(oracle_mod, max_distance):
    from nan_b200 import scenes

    ref = ov.ReferenceCaster("bvh")
    if not ref.available:
        pytest.skip("reference caster not built (oracle/_ref)")
    node = scenes.terrain_boxes(seed=7, grid=65, boxes=40)
    orc = oracle_mod.OracleScene(**node.pack())
    positions, indices = ov.world_geometry(orc.world_triangles())
    sites, normals = _sites(node, 384, seed=3)
    normals[:4] = 0.0  # the caster's zero-normal path: (0,0,1) and a nudged origin
    expect, stats = ref.cast(positions, indices, sites, normals, 512, max_distance, 1e-3, thread_count=4)
    got, counts = ov.visibility_sh16(orc, sites, normals, 512, max_distance, 1e-3)
    m = ov.compare(expect, got, 512)
    # the scalar layout runs the same watertight test family: every sample's
    # visible count and all 16 SH sums agree bit for bit
    assert stats["visible"] == int(counts.sum()), m
    assert m["samples_with_visible_count_difference"] == 0, m
    assert m["samples_with_identical_sh16"] == m["samples"], m


def test_reference_layouts_disagree_by_a_few_rays(oracle_mod):
    """The reference's own two layouts (scalar BVH and the AVX2 BVH8_CPU,
    whose SIMD triangle test rounds differently) differ by a ray or two per
    sample; the oracle matches the scalar layout exactly and differs from
    BVH8_CPU by the same margin."""
    from nan_b200 import scenes

    scalar, wide = ov.ReferenceCaster("bvh"), ov.ReferenceCaster("bvh8")
    if not (scalar.available and wide.available and wide.layout == 1):
        pytest.skip("reference BVH8_CPU caster not built")
    node = scenes.terrain_boxes(seed=7, grid=65, boxes=40)
    orc = oracle_mod.OracleScene(**node.pack())
    positions, indices = ov.world_geometry(orc.world_triangles())
    sites, normals = _sites(node, 384, seed=3)
    a, _ = scalar.cast(positions, indices, sites, normals, 512, 1000.0, 1e-3, thread_count=4)
    b, _ = wide.cast(positions, indices, sites, normals, 512, 1000.0, 1e-3, thread_count=4)
    got, _ = ov.visibility_sh16(orc, sites, normals, 512, 1000.0, 1e-3)
    between = ov.compare(a, b, 512)
    ours = ov.compare(b, got, 512)
    assert between["max_visible_count_difference"] <= 2 and ours["max_visible_count_difference"] <= 2
    assert ov.compare(a, got, 512)["samples_with_identical_sh16"] == 384
