"""Deficit repair and support estimate on the oracle (CPU) against the
reference's own Python deficit_repair_python and estimate_support_python
run on the same inputs (tests/golden): the repair cases of
test_surface_probes.py:436-600 (the budget, the zero-score skip) and a
seeded two-instance case give the same choices, counts, weight sums and
effective sample sizes; the support estimate gives the same f and m on a
flat and a tilted instance."""

import numpy as np
import pytest


@pytest.mark.parametrize("case", [0, 1, 2])
def test_repair_oracle_matches_reference(golden, case):
    from oracle.oracle import deficit_repair

    g = lambda name: golden[f"rep{case}_{name}"]
    mg, budget = (int(x) for x in g("params"))
    r = deficit_repair(g("bp"), g("bn"), g("bi"), g("cp"), g("cn"), g("ci"), g("ap"), g("an"), g("ai"), g("radii"),
                       min_gather_count=mg, max_repair_count=budget)
    np.testing.assert_array_equal(r["selected"], g("selected"))
    for name in ("counts_before", "counts_after", "weight_sums_before", "weight_sums_after", "ess_before",
                 "ess_after"):
        np.testing.assert_array_equal(r[name], g(name))
    if case == 1:  # the zero-score candidate is skipped, the repair goes on
        np.testing.assert_array_equal(r["counts_after"], [4, 4])
        assert r["selected"].shape[0] == 5


def test_repair_oracle_no_deficit_and_budget_cap(golden):
    from oracle.oracle import deficit_repair

    up = np.tile(np.float32([0, 1, 0]), (4, 1))
    pos = np.float32([[-0.15, 0, 0], [-0.05, 0, 0], [0.05, 0, 0], [0.15, 0, 0]])
    r = deficit_repair(pos, up, np.zeros(4), np.float32([[0.3, 0, 0]]), up[:1], np.zeros(1),
                       np.float32([[0, 0, 0]]), up[:1], np.zeros(1), [0.5], min_gather_count=4, max_repair_count=1)
    assert r["selected"].shape[0] == 0
    g = lambda name: golden[f"rep0_{name}"]
    r = deficit_repair(g("bp"), g("bn"), g("bi"), g("cp"), g("cn"), g("ci"), g("ap"), g("an"), g("ai"), g("radii"),
                       min_gather_count=4, max_repair_count=1)
    assert r["selected"].shape[0] == 1 and np.any(r["counts_after"] < 4)


def test_support_oracle_matches_reference(golden):
    """The support estimate equals the reference's Python
    estimate_support_python bit for bit, on a flat and a tilted instance."""
    from oracle.oracle import estimate_support

    g = lambda name: golden[f"sup_{name}"]
    f, m = estimate_support(g("rp"), g("rn"), g("ri"), g("ra"), g("qp"), g("qn"), g("qi"), g("radii"))
    np.testing.assert_array_equal(f, g("f"))
    np.testing.assert_array_equal(m, g("m"))
    assert f.min() < 0.6 and f.max() == 1.0  # border sites see less surface than interior ones


def test_support_oracle_matches_reference_dense(golden):
    """Queries that sum 10^4 to 2.5 x 10^4 terms: numpy's float32-to-float64
    sum runs through 8192-element buffers, and the oracle equals it."""
    from oracle.oracle import estimate_support

    g = lambda name: golden[f"supd_{name}"]
    f, m = estimate_support(g("rp"), g("rn"), g("ri"), g("ra"), g("qp"), g("qn"), g("qi"), g("radii"))
    np.testing.assert_array_equal(f, g("f"))
    np.testing.assert_array_equal(m, g("m"))


@pytest.mark.parametrize("case", ["sup", "supd"])
def test_support_oracle_against_reference_cpp(golden, case):
    """The reference's C++ estimate sums in grid-visit order; its own tests
    hold it to the Python form within 1e-6 (f) and 1e-5 (m)
    (test_surface_probes.py:806-816), and so does the oracle."""
    from oracle import ref_sampler
    from oracle.oracle import estimate_support

    if not ref_sampler.available():
        pytest.skip("reference sampler library not built")
    args = [golden[f"{case}_{k}"] for k in ("rp", "rn", "ri", "ra", "qp", "qn", "qi", "radii")]
    f, m = estimate_support(*args)
    cf, cm = ref_sampler.estimate_support(*args)
    np.testing.assert_allclose(f, cf, atol=1e-6)
    np.testing.assert_allclose(m, cm, atol=1e-5)


@pytest.mark.parametrize("case", [0, 1, 2])
def test_repair_oracle_against_reference_cpp(golden, case):
    """The reference's default (C++) repair, compiled from its sources: the
    same choices and counts; weight sums and ESS within the reference's own
    cross-backend bar (rtol 1e-6, test_surface_probes.py:469-495)."""
    from oracle import ref_sampler
    from oracle.oracle import deficit_repair

    if not ref_sampler.available():
        pytest.skip("reference sampler library not built")
    args = [golden[f"rep{case}_{n}"] for n in ("bp", "bn", "bi", "cp", "cn", "ci", "ap", "an", "ai", "radii")]
    mg, budget = (int(v) for v in golden[f"rep{case}_params"])
    mine = deficit_repair(*args, min_gather_count=mg, max_repair_count=budget)
    ref = ref_sampler.deficit_repair(*args, min_gather_count=mg, max_repair_count=budget)
    np.testing.assert_array_equal(mine["selected"], ref["selected"])
    for name in ("counts_before", "counts_after"):
        np.testing.assert_array_equal(mine[name], ref[name])
    for name in ("weight_sums_before", "weight_sums_after", "ess_before", "ess_after"):
        np.testing.assert_allclose(mine[name], ref[name], rtol=1e-6)
