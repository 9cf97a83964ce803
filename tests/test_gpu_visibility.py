"""GPU PMR visibility caster (nan_visibility_sh16) against the oracle and
against the reference's own compiled caster.

* Bit-exact with the oracle's restatement of the caster loop (same rays, the
  oracle's watertight any-hit, the caster's SH summation order), including
  samples with a zero normal (nudged origins) and both a short (0.5, the
  reference default) and a long ray length.
* On config 2's seeded 200,688-triangle scene (313x313 terrain + 500 boxes),
  4,096 surface samples x 512 rays: identical per-sample visible counts and
  SH16 to the reference's scalar-BVH caster (vbake_pmr_visibility_sh_tinybvh,
  layout 0, which runs the same watertight test family), with the reference
  benchmark's comparison (benchmark_tinybvh_visibility.py:45-61).
"""

import numpy as np
import pytest

from oracle import visibility as ov

pytestmark = pytest.mark.gpu


def _sites(node, count, seed):
    from nan_b200 import scenes

    probes, _ = scenes.surface_sites(node, count, seed=seed, double_sided_backs=False)
    return (np.ascontiguousarray(probes["position_radius"][:, :3]),
            np.ascontiguousarray(probes["normal_side"][:, :3]))


@pytest.mark.parametrize("max_distance,rays", [(1000.0, 512), (0.5, 512), (1000.0, 100)])
def test_gpu_visibility_equals_oracle(device, oracle_mod, max_distance, rays):
    import nan_b200
    from nan_b200 import scenes

    node = scenes.terrain_boxes(seed=7, grid=65, boxes=40)
    scene = nan_b200.Scene(device, node)
    orc = oracle_mod.OracleScene(**scene.host)
    sites, normals = _sites(node, 512, seed=3)
    normals[:5] = 0.0
    normals[5] = np.nan
    sh, counts = nan_b200.trace_pmr_visibility_sh(scene, sites, normals, ray_count=rays,
                                                  max_distance=max_distance, self_bias=1e-3)
    expect, expect_counts = ov.visibility_sh16(orc, sites, normals, rays, max_distance, 1e-3)
    np.testing.assert_array_equal(counts.cpu().numpy(), expect_counts)
    np.testing.assert_array_equal(sh.cpu().numpy().view(np.uint32), expect.view(np.uint32))
    device.check()


def test_gpu_visibility_equals_reference_caster_on_config2(device):
    import nan_b200
    from nan_b200 import scenes

    ref = ov.ReferenceCaster("bvh")
    if not ref.available:
        pytest.skip("reference caster not built (oracle/_ref)")
    node = scenes.terrain_boxes(seed=1, grid=313, boxes=500)
    scene = nan_b200.Scene(device, node)
    assert scene.triangle_count == 200_688
    positions, indices = ov.world_geometry(scene.world_triangles().cpu().numpy())
    sites, normals = _sites(node, 4096, seed=11)
    sampler = nan_b200.PMRVisibilitySHSampler(device)
    got = sampler.sample(scene, sites, normals, ray_count=512, max_distance=1000.0, self_bias=1e-3)
    expect, stats = ref.cast(positions, indices, sites, normals, 512, 1000.0, 1e-3)
    m = ov.compare(expect, got.cpu().numpy(), 512)
    assert m["samples_with_exact_visible_count"] >= 0.9999 * m["samples"], m
    assert m["samples_with_identical_sh16"] >= 0.9999 * m["samples"], m
    assert int(sampler.visible_counts.sum().item()) == stats["visible"] or m["samples_with_visible_count_difference"]
    device.check()
