"""Audit/repair candidate filter on the GPU against the oracle (and so the
reference's Python form through the golden vectors) and against the
reference's own C++ filter compiled from its sources: the reference case,
random candidates with exact duplicates, many sets in one call, and a
400k-candidate case."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [0, 1])
def test_filter_matches_golden(golden, device, case):
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    g = lambda name: golden[f"flt{case}_{name}"]
    pos, nrm = g("positions"), g("normals")
    res = SurfaceProbeSampler(device).filter_audit_repair_candidates(
        pos, nrm, pos, nrm, g("selected_base"), audit_cell_size=float(g("cell")[0]), normal_cosine_threshold=0.5)
    np.testing.assert_array_equal(res.audit_indices, g("audit"))
    np.testing.assert_array_equal(res.repair_indices, g("repair"))


def _random(n, seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-20)
    p[n // 2:], nrm[n // 2:] = p[:n // 2], nrm[:n // 2]
    return p, nrm


@pytest.mark.parametrize("n,cell", [(20000, 0.02), (20000, 0.5), (400000, 0.01)])
def test_filter_matches_oracle_and_reference_cpp(device, n, cell):
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler
    from oracle import ref_sampler
    from oracle.oracle import filter_audit_repair

    p, nrm = _random(n, seed=n + int(cell * 100))
    base_p, base_n = p[::2].copy(), nrm[::2].copy()
    sel = np.arange(0, base_p.shape[0], 3, dtype=np.uint32)
    sampler = SurfaceProbeSampler(device)
    sampler.filter_audit_repair_candidates(p[:64], nrm[:64], base_p, base_n, sel, audit_cell_size=cell,
                                           normal_cosine_threshold=0.5)
    t0 = time.perf_counter()
    res = sampler.filter_audit_repair_candidates(p, nrm, base_p, base_n, sel, audit_cell_size=cell,
                                                 normal_cosine_threshold=0.5)
    gpu_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    audit, repair = filter_audit_repair(p, nrm, base_p, base_n, sel, audit_cell_size=cell, normal_cosine_threshold=0.5)
    cpu_s = time.perf_counter() - t0
    print(f"filter n {n} cell {cell}: audit {audit.shape[0]} repair {repair.shape[0]} gpu {gpu_s * 1e3:.1f} ms "
          f"(host arrays in and out) oracle {cpu_s * 1e3:.1f} ms")
    np.testing.assert_array_equal(res.audit_indices, audit)
    np.testing.assert_array_equal(res.repair_indices, repair)
    if ref_sampler.available():
        ra, rr = ref_sampler.filter_audit_repair_candidates(p, nrm, base_p, base_n, sel, audit_cell_size=cell,
                                                            normal_cosine_threshold=0.5)
        np.testing.assert_array_equal(res.audit_indices, ra)
        np.testing.assert_array_equal(res.repair_indices, rr)
    device.check()


def test_filter_sets_in_one_call(device):
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler
    from oracle.oracle import filter_audit_repair

    rng = np.random.default_rng(12)
    sizes = rng.integers(1, 3000, 37)
    cells = rng.uniform(0.01, 0.2, 37)
    pos, nrm = _random(int(sizes.sum()), seed=3)
    sets = np.repeat(np.arange(37, dtype=np.uint32), sizes)
    sel = np.flatnonzero(rng.random(pos.shape[0]) < 0.1).astype(np.uint32)
    res = SurfaceProbeSampler(device).filter_audit_repair_candidates(
        pos, nrm, pos, nrm, sel, audit_cell_size=cells, normal_cosine_threshold=0.5, candidate_sets=sets,
        base_sets=sets)
    audit, repair = filter_audit_repair(pos, nrm, pos, nrm, sel, audit_cell_size=cells, normal_cosine_threshold=0.5,
                                        candidate_sets=sets, base_sets=sets)
    np.testing.assert_array_equal(res.audit_indices, audit)
    np.testing.assert_array_equal(res.repair_indices, repair)
    device.check()


def test_filter_rejects_bad_inputs(device):
    from nan_b200.surface_probe_sampler import SurfaceProbeSampler

    p, nrm = _random(100, seed=1)
    sampler = SurfaceProbeSampler(device)
    with pytest.raises(Exception, match="invalid index"):
        sampler.filter_audit_repair_candidates(p, nrm, p, nrm, [5, 100], audit_cell_size=0.1,
                                               normal_cosine_threshold=0.5)
    bad = p.copy()
    bad[3, 1] = np.inf
    with pytest.raises(Exception, match="finite"):
        sampler.filter_audit_repair_candidates(bad, nrm, p, nrm, [0], audit_cell_size=0.1,
                                               normal_cosine_threshold=0.5)
    with pytest.raises(Exception, match="cell size"):
        sampler.filter_audit_repair_candidates(p, nrm, p, nrm, [0], audit_cell_size=0.0,
                                               normal_cosine_threshold=0.5)
    device.check()
