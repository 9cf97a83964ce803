"""Weighted sample elimination on the GPU (parallel rounds) against the
oracle's one-at-a-time elimination: identical survivors on the reference's
golden candidate sets, on a batch of 40 uneven sets in one call and on a
200k-candidate terrain set; the adaptive (density-driven) elimination on
the reference's golden cases and 40 sets with varying densities; and the WSE site layout of the terrain (5x
oversampling) spaces its sites wider than area-weighted random sites while
keeping every octree range valid."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_wse_matches_oracle_on_reference_cases(golden, device):
    from nan_b200.surface_probe_sampler import weighted_sample_elimination
    from oracle.oracle import wse_eliminate

    for case in range(3):
        pos, nrm = golden[f"wse{case}_positions"], golden[f"wse{case}_normals"]
        count, area = golden[f"wse{case}_params"]
        sel, radius = weighted_sample_elimination(pos, nrm, int(count), surface_area=float(area), device=device)
        keep, radii, _ = wse_eliminate(pos, nrm, [0, pos.shape[0]], [int(count)], [area])
        np.testing.assert_array_equal(sel, np.flatnonzero(keep))
        assert radius == float(radii[0])


@pytest.mark.parametrize("case", [0, 1, 2])
def test_adaptive_matches_oracle_on_reference_cases(golden, device, case):
    """The adaptive elimination: the oracle's survivors (which are the
    reference Python's on cases 0 and 1) and the base Poisson radius."""
    from nan_b200.surface_probe_sampler import adaptive_weighted_sample_elimination
    from oracle.oracle import wse_eliminate

    g = lambda name: golden[f"awse{case}_{name}"]
    pos, nrm, dens = g("positions"), g("normals"), g("densities")
    count, area = g("params")
    sel, radius = adaptive_weighted_sample_elimination(pos, nrm, dens, int(count), surface_area=float(area),
                                                       partition_masses=np.ones_like(dens), device=device)
    keep, radii, _ = wse_eliminate(pos, nrm, [0, pos.shape[0]], [int(count)], [area], relative_densities=dens)
    np.testing.assert_array_equal(sel, np.flatnonzero(keep))
    assert radius == float(radii[0])
    if case < 2:
        np.testing.assert_array_equal(sel, g("selected"))


def test_adaptive_batches_match_oracle(device):
    """40 uneven sets on terrain + boxes with densities varying 6:1 across
    each set, one call."""
    from nan_b200 import scenes
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler
    from oracle.oracle import wse_eliminate

    node = scenes.terrain_boxes(seed=2, grid=129, boxes=40)
    pos, nrm, off, outs, areas = _surface_candidates(node, 40.0, seed=9)
    rng = np.random.default_rng(4)
    dens = (0.4 + 2.0 * (0.5 + 0.5 * np.sin(pos[:, 0] * 0.7 + pos[:, 2] * 0.3))
            * rng.uniform(0.9, 1.1, pos.shape[0])).astype(np.float32)
    sampler = SurfaceProbeSampler(device)
    t0 = time.perf_counter()
    keep, radii = sampler.eliminate(pos, nrm, off, outs, areas, relative_densities=dens)
    keep = keep.cpu().numpy()
    gpu_s = time.perf_counter() - t0
    ref, ref_radii, _ = wse_eliminate(pos, nrm, off, outs, areas, relative_densities=dens)
    print(f"adaptive sets {len(outs)} candidates {pos.shape[0]} rounds {sampler.last_rounds} "
          f"gpu {gpu_s * 1e3:.1f} ms")
    np.testing.assert_array_equal(keep, ref)
    np.testing.assert_array_equal(radii, ref_radii)
    device.check()


def test_adaptive_rejects_bad_densities(device):
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    pos = np.random.default_rng(1).uniform(0, 1, (100, 3)).astype(np.float32)
    nrm = np.tile(np.float32([0, 1, 0]), (100, 1))
    dens = np.ones(100, np.float32)
    dens[17] = 0.0
    with pytest.raises(Exception, match="densities"):
        SurfaceProbeSampler(device).eliminate(pos, nrm, [0, 100], [20], [1.0], relative_densities=dens)
    device.check()


def _surface_candidates(node, per_instance_scale, seed):
    rng = np.random.default_rng(seed)
    pos, nrm, off, outs, areas = [], [], [0], [], []
    for mesh_id, _, transform_id in node.instances:
        mesh = node.meshes[mesh_id]
        m = node.transforms[transform_id].astype(np.float64)
        p = mesh.vertices[:, :3].astype(np.float64) @ m[:3, :3].T + m[:3, 3]
        t = p[mesh.indices.astype(np.int64).reshape(-1, 3)]
        cr = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
        a = 0.5 * np.linalg.norm(cr, axis=1)
        k = max(5, int(a.sum() * per_instance_scale))
        ch = rng.choice(t.shape[0], size=k, p=a / a.sum())
        u = rng.random((k, 2))
        su = np.sqrt(u[:, 0])
        b1, b2 = su * (1 - u[:, 1]), su * u[:, 1]
        pos.append((t[ch, 0] + (t[ch, 1] - t[ch, 0]) * b1[:, None] + (t[ch, 2] - t[ch, 0]) * b2[:, None]))
        nrm.append(cr[ch] / np.linalg.norm(cr[ch], axis=1, keepdims=True))
        off.append(off[-1] + k)
        outs.append(max(1, k // 5))
        areas.append(a.sum())
    return (np.concatenate(pos).astype(np.float32), np.concatenate(nrm).astype(np.float32), np.array(off),
            np.array(outs), np.array(areas, np.float32))


@pytest.mark.parametrize("boxes,scale", [(40, 40.0), (0, 90.0)])
def test_wse_batches_match_oracle(device, boxes, scale):
    from nan_b200 import scenes
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler
    from oracle.oracle import wse_eliminate

    node = scenes.terrain_boxes(seed=2, grid=129 if boxes else 313, boxes=boxes)
    pos, nrm, off, outs, areas = _surface_candidates(node, scale, seed=5)
    sampler = SurfaceProbeSampler(device)
    t0 = time.perf_counter()
    keep, radii = sampler.eliminate(pos, nrm, off, outs, areas)
    keep = keep.cpu().numpy()
    gpu_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref, ref_radii, _ = wse_eliminate(pos, nrm, off, outs, areas)
    cpu_s = time.perf_counter() - t0
    print(f"sets {len(outs)} candidates {pos.shape[0]} rounds {sampler.last_rounds} gpu {gpu_s * 1e3:.1f} ms "
          f"oracle {cpu_s * 1e3:.1f} ms")
    np.testing.assert_array_equal(keep, ref)
    np.testing.assert_array_equal(radii, ref_radii)
    for k in range(len(outs)):
        assert int(keep[off[k]:off[k + 1]].sum()) == min(int(outs[k]), int(off[k + 1] - off[k]))
    device.check()


def test_wse_layout_spaces_sites_wider_than_random(device):
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout

    node = scenes.terrain_boxes(seed=1, grid=129, boxes=0)
    prof = {}
    wse = SurfaceProbeSiteLayout.build_wse(node, 4000, device=device, seed=3, profile=prof, repair_min_gather=0,
                                           adaptive_wse=False)
    rnd = SurfaceProbeSiteLayout.build(node, 4000, seed=3)
    print("wse layout", prof)

    def spacing(layout):
        p = layout.probes["position_radius"][:, :3].astype(np.float64)
        from scipy.spatial import cKDTree

        d, _ = cKDTree(p).query(p, k=2)
        return float(d[:, 1].mean()), float(d[:, 1].min())

    sw, sr = spacing(wse), spacing(rnd)
    print("mean / min nearest distance: wse", sw, "random", sr)
    assert wse.total_probe_count == rnd.total_probe_count
    assert sw[0] > 1.2 * sr[0] and sw[1] > 3.0 * sr[1]
    info = wse.instance_infos[0]
    found = wse.query_probe_indices(0, info.root_center, radius=info.root_extent * 4.0)
    np.testing.assert_array_equal(np.sort(found), np.arange(info.probe_offset, info.probe_offset + info.probe_count))


def test_wse_layout_repair_fills_gather_deficits(device):
    """With boxes on the terrain, the repair adds sites where audit points
    gather fewer than 4 (box faces, seams) and every audit deficit it can
    reach is closed."""
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout

    node = scenes.terrain_boxes(seed=2, grid=97, boxes=40)
    prof = {}
    layout = SurfaceProbeSiteLayout.build_wse(node, 3000, device=device, seed=5, profile=prof)
    print("repair", prof)
    assert 0 < prof["repair_sites"] <= 900
    assert prof["audits_below_min_after_repair"] < prof["audits_below_min_before"]
    assert prof["audits_below_min_after"] == 0 and prof["zero_gather_after"] == 0
    fronts = int(((layout.probes["meta"][:, 3] & 1) == 0).sum())
    assert fronts == prof["base_sites"] + prof["repair_sites"] + prof["protected_sites"]
    for k, info in enumerate(layout.instance_infos):
        if info.probe_count:
            found = layout.query_probe_indices(k, info.root_center, radius=info.root_extent * 4.0)
            assert found.shape[0] == info.probe_count


def test_adaptive_layout_reallocates_without_changing_base_budget(device):
    """test_surface_probes.py:1068-1090 on the reference's demo box: the
    density prepass moves sites between instances, the base budget stays 80."""
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout

    node = scenes.reference_demo()
    pa, pu = {}, {}
    adaptive = SurfaceProbeSiteLayout.build_wse(node, 80, oversample_factor=3, seed=7, repair_min_gather=0,
                                                device=device, profile=pa)
    uniform = SurfaceProbeSiteLayout.build_wse(node, 80, oversample_factor=3, seed=7, repair_min_gather=0,
                                               adaptive_wse=False, device=device, profile=pu)
    assert pa["adaptive"] and not pu["adaptive"]
    assert pa["base_sites"] == 80 and pu["base_sites"] == 80
    assert adaptive.adaptive_wse and not uniform.adaptive_wse
    assert adaptive.total_base_surface_site_count == 80 and uniform.total_base_surface_site_count == 80
    counts = lambda layout: [info.base_surface_site_count for info in layout.instance_infos]
    print("adaptive", counts(adaptive), "uniform", counts(uniform))
    assert counts(adaptive) != counts(uniform)


def test_adaptive_layout_densifies_low_support_surface(device):
    """Where the kernel disc leaves the surface (the terrain's border, the
    boxes) support is low and the density multiplier high: the adaptive
    layout puts a larger share of the sites there than the uniform one."""
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout

    node = scenes.terrain_boxes(seed=2, grid=97, boxes=40)
    kw = dict(device=device, seed=5, repair_min_gather=0)
    pa = {}
    adaptive = SurfaceProbeSiteLayout.build_wse(node, 3000, profile=pa, **kw)
    uniform = SurfaceProbeSiteLayout.build_wse(node, 3000, adaptive_wse=False, **kw)
    print("adaptive profile", pa)

    def shares(layout):
        front = (layout.probes["meta"][:, 3] & 1) == 0
        inst = layout.probes["meta"][front, 3] >> 8
        pos = layout.probes["position_radius"][front, :3]
        half = 0.5 * 0.15 * 96
        radius = float(layout.instance_infos[0].kernel_radius)
        on_terrain = inst == 0
        border = on_terrain & ((np.abs(pos[:, 0]) > half - radius) | (np.abs(pos[:, 2]) > half - radius))
        return float((~on_terrain).mean()), float(border.sum() / max(on_terrain.sum(), 1))

    (box_a, border_a), (box_u, border_u) = shares(adaptive), shares(uniform)
    print("box share adaptive / uniform", box_a, box_u, "border share", border_a, border_u)
    assert box_a > box_u and border_a > border_u


def test_protected_closure_eliminates_unbudgeted_gather_deficits(device):
    """test_surface_probes.py:1001-1032: with no repair budget and a small
    kernel, audit points stay short after the repair; the closure adds
    colocated protected sites (at most 4 per short audit point) until none
    is short, and the build repeats exactly."""
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import SurfaceProbeSiteLayout
    from nan_b200.surface_probe_resources import SURFACE_PROBE_FLAG_PROTECTED

    node = scenes.reference_demo()
    options = dict(oversample_factor=1, seed=7, kernel_radius_scale=0.5, repair_budget_ratio=0.0, device=device)
    prof = {}
    layout = SurfaceProbeSiteLayout.build_wse(node, 8, profile=prof, **options)
    print("closure", prof)
    assert prof["repair_sites"] == 0
    assert prof["audits_below_min_after_repair"] > 0
    assert prof["protected_sites"] > 0
    assert prof["audits_below_min_after"] == 0 and prof["zero_gather_after"] == 0
    assert prof["protected_sites"] <= 4 * prof["audits_below_min_after_repair"]
    protected = (layout.probes["meta"][:, 3] & SURFACE_PROBE_FLAG_PROTECTED) != 0
    assert protected.any()
    # the reference's layout statistics (test_surface_probes.py:1010-1022)
    assert layout.total_repair_surface_site_count == 0
    assert layout.zero_gather_after_repair > 0 and layout.deficit_point_count_after_repair > 0
    assert layout.total_protected_surface_site_count == prof["protected_sites"] > 0
    assert layout.zero_gather_after == 0 and layout.deficit_point_count_after == 0
    assert layout.total_protected_surface_site_count <= layout.deficit_point_count_after_repair * 4
    assert layout.total_surface_site_count == 8 + layout.total_protected_surface_site_count
    assert sum(i.protected_surface_site_count for i in layout.instance_infos) == prof["protected_sites"]
    assert sum(i.base_surface_site_count for i in layout.instance_infos) == 8
    again = SurfaceProbeSiteLayout.build_wse(node, 8, **options)
    np.testing.assert_array_equal(again.probes, layout.probes)


def test_density_mode_makes_base_population_an_output(device):
    """test_surface_probes.py:889-914 through the reference's class name and
    keywords: in density mode the base site count is an output, at least the
    floor of 4 per instance, and the sum of the instances' counts; a larger
    density scale places more sites."""
    from nan_b200 import scenes
    from nan_b200.surface_probe_layout import SurfaceProbeLayout

    node = scenes.reference_demo()
    kw = dict(target_probe_count=None, adaptive_mass_site_density=0.5, density_reference_kernel_radius=2.5,
              oversample_factor=1, seed=7, repair_budget_ratio=0.0, device=device)
    layout = SurfaceProbeLayout.build(node, density_scale=1.0, **kw)
    assert isinstance(layout, SurfaceProbeLayout)
    assert layout.density_driven and layout.density_scale == 1.0
    assert layout.total_surface_area > 0.0 and layout.total_adaptive_mass > 0.0
    assert layout.total_base_surface_site_count >= 4 * len(layout.instance_infos)
    assert layout.total_base_surface_site_count == sum(i.base_surface_site_count for i in layout.instance_infos)
    denser = SurfaceProbeLayout.build(node, density_scale=16.0, **kw)
    assert denser.total_base_surface_site_count > layout.total_base_surface_site_count
    with pytest.raises(ValueError):
        SurfaceProbeLayout.build(node, target_probe_count=None, device=device)
