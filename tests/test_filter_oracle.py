"""Audit/repair candidate filter on the oracle (CPU), pinned to the
reference's Python form (_deduplicate_audit_candidates and
_exclude_selected_duplicates, surface_probes.py:782-832) through the golden
vectors and to its default C++ form (surface_probe_sampler.cpp:1736-1997),
compiled from the reference's sources, on random candidates with exact
duplicates; plus batching of several sets."""

import numpy as np
import pytest


@pytest.mark.parametrize("case", [0, 1])
def test_oracle_equals_reference_python(golden, case):
    from oracle.oracle import filter_audit_repair

    g = lambda name: golden[f"flt{case}_{name}"]
    pos, nrm = g("positions"), g("normals")
    audit, repair = filter_audit_repair(pos, nrm, pos, nrm, g("selected_base"), audit_cell_size=float(g("cell")[0]),
                                        normal_cosine_threshold=0.5)
    np.testing.assert_array_equal(audit, g("audit"))
    np.testing.assert_array_equal(repair, g("repair"))


def test_reference_case():
    """test_surface_probes.py:697-730: cell, normal and exact-duplicate rules."""
    from oracle.oracle import filter_audit_repair

    p = np.float32([[0.0, 0, 0], [0.1, 0, 0], [0.0, 0, 0], [0.2, 0, 0], [1.1, 0, 0]])
    n = np.float32([[0, 1, 0], [0, 1, 0], [0, 1, 0], [0, -1, 0], [0, 1, 0]])
    audit, repair = filter_audit_repair(p, n, p, n, [0], audit_cell_size=1.0, normal_cosine_threshold=0.5)
    np.testing.assert_array_equal(audit, [0, 3, 4])
    np.testing.assert_array_equal(repair, [1, 3, 4])


@pytest.mark.parametrize("cell", [0.02, 0.05, 0.5])
def test_oracle_equals_reference_cpp(cell):
    from oracle import ref_sampler
    from oracle.oracle import filter_audit_repair

    if not ref_sampler.available():
        pytest.skip("reference sampler library not built")
    rng = np.random.default_rng(int(cell * 1000))
    n = 20000
    p = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-20)
    p[n // 2:], nrm[n // 2:] = p[:n // 2], nrm[:n // 2]
    base_p, base_n = p[::2].copy(), nrm[::2].copy()
    sel = np.arange(0, base_p.shape[0], 3, dtype=np.uint32)
    mine = filter_audit_repair(p, nrm, base_p, base_n, sel, audit_cell_size=cell, normal_cosine_threshold=0.5)
    ref = ref_sampler.filter_audit_repair_candidates(p, nrm, base_p, base_n, sel, audit_cell_size=cell,
                                                     normal_cosine_threshold=0.5)
    np.testing.assert_array_equal(mine[0], ref[0])
    np.testing.assert_array_equal(mine[1], ref[1])


def test_sets_filter_independently():
    from oracle.oracle import filter_audit_repair

    rng = np.random.default_rng(3)
    sizes, cells = [500, 800, 300], [0.05, 0.1, 0.02]
    parts = []
    for k, n in enumerate(sizes):
        p = rng.uniform(0, 1, (n, 3)).astype(np.float32)
        nrm = rng.normal(size=(n, 3)).astype(np.float32)
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        p[n // 2:], nrm[n // 2:] = p[:n // 2], nrm[:n // 2]
        parts.append((p, nrm))
    # the same points in two sets are not duplicates of each other
    parts[2] = (parts[0][0][:300].copy(), parts[0][1][:300].copy())
    pos = np.concatenate([q[0] for q in parts])
    nrm = np.concatenate([q[1] for q in parts])
    sets = np.repeat(np.arange(3, dtype=np.uint32), sizes)
    offsets = np.concatenate([[0], np.cumsum(sizes)])
    sel = np.concatenate([np.arange(offsets[k], offsets[k] + 60, 7) for k in range(3)]).astype(np.uint32)
    audit, repair = filter_audit_repair(pos, nrm, pos, nrm, sel, audit_cell_size=cells, normal_cosine_threshold=0.5,
                                        candidate_sets=sets, base_sets=sets)
    for k in range(3):
        b, e = offsets[k], offsets[k + 1]
        local_sel = sel[(sel >= b) & (sel < e)] - b
        a_k, r_k = filter_audit_repair(pos[b:e], nrm[b:e], pos[b:e], nrm[b:e], local_sel, audit_cell_size=cells[k],
                                       normal_cosine_threshold=0.5)
        np.testing.assert_array_equal(audit[(audit >= b) & (audit < e)] - b, a_k)
        np.testing.assert_array_equal(repair[(repair >= b) & (repair < e)] - b, r_k)
