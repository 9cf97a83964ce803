"""Deficit repair on the GPU (parallel rounds) against the oracle's
one-at-a-time repair: the same choices in the same order, the same counts,
weight sums and effective sample sizes, on the reference's cases and on a
seeded 12-instance case with 30k audits and 20k candidates."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _compare(gpu, ref):
    np.testing.assert_array_equal(gpu.selected_candidate_indices, ref["selected"])
    for name in ("counts_before", "counts_after", "weight_sums_before", "weight_sums_after", "ess_before",
                 "ess_after"):
        np.testing.assert_array_equal(getattr(gpu, name), ref[name])


def test_repair_matches_oracle_on_reference_cases(golden, device):
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler
    from oracle.oracle import deficit_repair

    sampler = SurfaceProbeSampler(device)
    for case in range(3):
        g = lambda name: golden[f"rep{case}_{name}"]
        mg, budget = (int(x) for x in g("params"))
        args = (g("bp"), g("bn"), g("bi"), g("cp"), g("cn"), g("ci"), g("ap"), g("an"), g("ai"), g("radii"))
        gpu = sampler.deficit_repair(*args, min_gather_count=mg, max_repair_count=budget)
        _compare(gpu, deficit_repair(*args, min_gather_count=mg, max_repair_count=budget))
        np.testing.assert_array_equal(gpu.selected_candidate_indices, g("selected"))
    device.check()


def test_repair_matches_oracle_at_scale(device):
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler
    from oracle.oracle import deficit_repair

    rng = np.random.default_rng(12)
    parts = {k: [] for k in ("bp", "bn", "bi", "cp", "cn", "ci", "ap", "an", "ai")}
    radii = []
    for inst in range(12):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        t = np.cross(n, [0.3, 0.5, 0.8])
        t /= np.linalg.norm(t)
        b = np.cross(n, t)
        origin = rng.uniform(-50, 50, 3)

        def sheet(count):
            u = rng.uniform(0, 6, (count, 2))
            return (origin + u[:, :1] * t + u[:, 1:] * b).astype(np.float32)

        for key, count in (("b", 150), ("c", 1700), ("a", 2500)):
            parts[key + "p"].append(sheet(count))
            parts[key + "n"].append(np.tile(n.astype(np.float32), (count, 1)))
            parts[key + "i"].append(np.full(count, inst, np.uint32))
        radii.append(0.45 + 0.05 * inst)
    args = [np.concatenate(parts[k]) for k in ("bp", "bn", "bi", "cp", "cn", "ci", "ap", "an", "ai")]
    args.append(np.asarray(radii, np.float32))
    sampler = SurfaceProbeSampler(device)
    sampler.deficit_repair(*args, min_gather_count=4, max_repair_count=600)  # first call: module load
    t0 = time.perf_counter()
    gpu = sampler.deficit_repair(*args, min_gather_count=4, max_repair_count=600)
    gpu_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref = deficit_repair(*args, min_gather_count=4, max_repair_count=600)
    cpu_s = time.perf_counter() - t0
    print(f"repairs {gpu.selected_candidate_indices.shape[0]} rounds {gpu.rounds} gpu {gpu_s * 1e3:.1f} ms "
          f"oracle {cpu_s * 1e3:.1f} ms; audits below 4 before {(gpu.counts_before < 4).sum()} "
          f"after {(gpu.counts_after < 4).sum()}")
    assert gpu.selected_candidate_indices.shape[0] > 100
    _compare(gpu, ref)
    device.check()


def test_support_matches_oracle(golden, device):
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler
    from oracle.oracle import estimate_support

    g = lambda name: golden[f"sup_{name}"]
    args = (g("rp"), g("rn"), g("ri"), g("ra"), g("qp"), g("qn"), g("qi"), g("radii"))
    f, m = SurfaceProbeSampler(device).estimate_support(*args)
    rf, rm = estimate_support(*args)
    np.testing.assert_array_equal(f, rf)
    np.testing.assert_array_equal(m, rm)
    np.testing.assert_array_equal(f, g("f"))


def test_support_dense_matches_golden(golden, device):
    """No cap on the terms of a query: 10^4 to 2.5 x 10^4 per site, summed in
    numpy's buffered pairwise order, equal to the reference's Python form."""
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    g = lambda name: golden[f"supd_{name}"]
    args = (g("rp"), g("rn"), g("ri"), g("ra"), g("qp"), g("qn"), g("qi"), g("radii"))
    f, m = SurfaceProbeSampler(device).estimate_support(*args)
    np.testing.assert_array_equal(f, g("f"))
    np.testing.assert_array_equal(m, g("m"))
    device.check()


def test_wse_layout_support_in_records(device):
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout

    node = scenes.terrain_boxes(seed=2, grid=97, boxes=40)
    prof = {}
    layout = SurfaceProbeSiteLayout.build_wse(node, 3000, device=device, seed=5, profile=prof)
    support = layout.probes["normal_side"][:, 3]
    print("support p10 / p50", prof["support_p10"], prof["support_p50"], "density p95", prof["density_p95"])
    assert support.min() > 0.0 and support.max() <= 1.0
    assert prof["support_p10"] < prof["support_p50"]


def test_wse_layout_support_flat_interior(device):
    """On a flat plane a site whose kernel disc lies inside the plane sees the
    whole flat-disc mass, so its support is near 1; sites at the border see
    about half of it."""
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout

    node = scenes.terrain_boxes(seed=3, grid=81, boxes=0, amplitude=0.0)
    layout = SurfaceProbeSiteLayout.build_wse(node, 3000, device=device, seed=9)
    radius = float(layout.instance_infos[0].kernel_radius)
    pos = layout.probes["position_radius"][:, :3]
    support = layout.probes["normal_side"][:, 3]
    half = 0.5 * 0.15 * 80
    inner = (np.abs(pos[:, 0]) < half - radius) & (np.abs(pos[:, 2]) < half - radius)
    edge = (np.abs(pos[:, 0]) > half - 0.1 * radius) | (np.abs(pos[:, 2]) > half - 0.1 * radius)
    assert inner.sum() > 1000 and edge.sum() > 10
    assert np.median(support[inner]) > 0.9 and np.percentile(support[inner], 10) > 0.6
    assert np.median(support[edge]) < 0.8
