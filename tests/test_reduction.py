"""Exact homogeneous-equality reduction: parity with the reference's plan on
seeded LPs (fixture generated from the reference by
``tests/golden/make_reduction_golden.py``) and the reference's own
known-answer cases (``tests/test_lp_equality_reduction.py``)."""
import numpy as np
import pytest
from scipy.sparse import csr_matrix

from co_cultivation_metabolic_atlas_b200.lp_trace import certificate
from co_cultivation_metabolic_atlas_b200.reduction import EqualityReduction
from tests.golden.make_reduction_golden import cases


def _p(a, rhs, lower, upper, c, neq):
    return (csr_matrix(np.asarray(a, float)), np.asarray(rhs, float), np.asarray(lower, float),
            np.asarray(upper, float), np.asarray(c, float), neq)


@pytest.mark.parametrize("name", ["species0", "species1", "species2", "chains"])
def test_plan_reduced_problem_and_lift_match_reference(golden_dir, name):
    g = np.load(golden_dir / "reduction_golden.npz")
    G = lambda k: g[f"{name}__{k}"]
    p = cases()[name]
    plan = EqualityReduction(p)
    red = plan.reduce(p)
    t = plan.transform.tocoo()
    ref_t = csr_matrix((G("t_val"), (G("t_row"), G("t_col"))), shape=plan.transform.shape)
    assert (plan.transform != ref_t).nnz == 0
    np.testing.assert_array_equal(plan.eliminated_rows, G("eliminated"))
    np.testing.assert_array_equal(plan.kept_rows, G("kept"))
    np.testing.assert_array_equal(plan.representatives, G("representatives"))
    ref_dl = csr_matrix((G("dl_val"), (G("dl_row"), G("dl_col"))), shape=plan.dual_lift_map.shape)
    assert abs(plan.dual_lift_map - ref_dl).max() <= 1e-15 if ref_dl.nnz else plan.dual_lift_map.nnz == 0
    ra, rrhs, rlo, rup, rc, rneq = red.problem
    np.testing.assert_array_equal(ra.indptr, G("ra_indptr"))
    np.testing.assert_array_equal(ra.indices, G("ra_indices"))
    np.testing.assert_array_equal(ra.data, G("ra_data"))
    for ours, key in ((rrhs, "rrhs"), (rlo, "rlo"), (rup, "rup"), (rc, "rc")):
        np.testing.assert_array_equal(ours, G(key))
    assert rneq == int(G("rneq"))
    np.testing.assert_array_equal(red.lower_witness, G("lower_witness"))
    np.testing.assert_array_equal(red.upper_witness, G("upper_witness"))
    y = red.lift_dual(G("ry"), G("rcost"))
    np.testing.assert_allclose(y, G("y"), rtol=0, atol=1e-12)


def test_equal_variables_reduce_and_lift_to_a_certified_original_pair():
    p = _p([[1.0, -1.0]], [0.0], [0.0, 0.0], [1.0, 1.0], [-1.0, -1.0], 1)
    plan = EqualityReduction(p)
    red = plan.reduce(p)
    np.testing.assert_array_equal(plan.eliminated_rows, [0])
    np.testing.assert_allclose(plan.transform.toarray(), [[1.0], [1.0]])
    assert red.problem[0].shape == (0, 1)
    np.testing.assert_allclose(red.problem[2:5], ([0.0], [1.0], [-2.0]))
    x = red.expand_primal([1.0])
    y = red.lift_dual(np.empty(0), [-2.0])
    np.testing.assert_allclose(x, [1.0, 1.0])
    np.testing.assert_allclose(y, [1.0])
    assert certificate(p, x, y)["certificate_passed"]


def test_scaled_relation_uses_the_largest_weight_as_representative():
    p = _p([[-2.0, 1.0]], [0.0], [0.0, 0.0], [1.0, 2.0], [-1.0, 0.0], 1)
    plan = EqualityReduction(p)
    red = plan.reduce(p)
    np.testing.assert_allclose(plan.transform.toarray(), [[0.5], [1.0]])
    np.testing.assert_array_equal(plan.representatives, [1])
    assert red.upper_witness.tolist() == [1]
    np.testing.assert_allclose(red.problem[3], [2.0])
    np.testing.assert_allclose(red.problem[4], [-0.5])
    np.testing.assert_allclose(red.allocate_bound_reduced_cost([-0.5]), [0.0, -0.5])
    y = red.lift_dual([], [-0.5])
    np.testing.assert_allclose(y, [0.5])
    assert certificate(p, red.expand_primal([2.0]), y)["certificate_passed"]


def test_negative_weight_maps_a_reduced_lower_bound_to_an_original_upper_bound():
    p = _p([[1.0, 1.0]], [0.0], [0.0, -1.0], [1.0, 0.0], [0.0, -1.0], 1)
    plan = EqualityReduction(p)
    red = plan.reduce(p)
    np.testing.assert_allclose(plan.transform.toarray(), [[1.0], [-1.0]])
    assert red.lower_witness.tolist() == [0]
    y = red.lift_dual([], [1.0])
    np.testing.assert_allclose(y, [-1.0])
    assert certificate(p, [0.0, 0.0], y)["certificate_passed"]


def test_tree_dual_map_inverts_the_eliminated_transpose():
    p = _p([[1.0, -1.0, 0.0], [0.0, 1.0, -1.0]], [0.0, 0.0], [-np.inf] * 3, [np.inf] * 3, [0.0] * 3, 2)
    plan = EqualityReduction(p)
    d = np.asarray([1.0, 0.0, -1.0])
    np.testing.assert_allclose(plan.transform.toarray(), [[1.0], [1.0], [1.0]])
    np.testing.assert_allclose(plan.dual_lift_map @ d, [1.0, 1.0])
    np.testing.assert_allclose(p[0].T @ (plan.dual_lift_map @ d), d)


def test_cycle_is_kept_while_a_spanning_forest_is_eliminated():
    p = _p([[1.0, -1.0, 0.0], [0.0, 1.0, -1.0], [-1.0, 0.0, 1.0]], [0.0] * 3, [0.0] * 3, [1.0] * 3, [0.0] * 3, 3)
    plan = EqualityReduction(p)
    red = plan.reduce(p)
    np.testing.assert_array_equal(plan.eliminated_rows, [0, 1])
    np.testing.assert_array_equal(plan.kept_rows, [2])
    assert red.problem[-1] == 1 and red.problem[0].shape == (1, 1) and red.problem[0].nnz == 0


def test_near_zero_coefficients_and_nonhomogeneous_rows_are_kept():
    assert EqualityReduction(_p([[1.0, -1e-12]], [0.0], [0.0, 0.0], [1.0, 1.0], [0.0, 0.0], 1)).eliminated_rows.size == 0
    assert EqualityReduction(_p([[1.0, -1.0]], [1.0], [0.0, 0.0], [2.0, 2.0], [0.0, 0.0], 1)).eliminated_rows.size == 0


def test_plan_is_fixed_by_the_equality_block_while_vectors_and_kept_rows_change():
    plan = EqualityReduction(_p([[1.0, -1.0], [2.0, 3.0]], [0.0, 8.0], [0.0, 0.0], [4.0, 4.0], [1.0, 2.0], 1))
    changed = _p([[1.0, -1.0], [4.0, -1.0]], [0.0, 7.0], [-1.0, 0.0], [3.0, 2.0], [-2.0, 5.0], 1)
    r = plan.reduce(changed).problem
    np.testing.assert_allclose(r[0].toarray(), [[3.0]])
    np.testing.assert_allclose(r[1:5], ([7.0], [0.0], [2.0], [3.0]))
    stale = list(changed)
    stale[0] = csr_matrix([[1.0, -2.0], [4.0, -1.0]])
    with pytest.raises(ValueError, match="fingerprint"):
        plan.reduce(tuple(stale))


def test_infeasible_bound_intersection_is_rejected():
    p = _p([[1.0, -1.0]], [0.0], [1.0, 0.0], [2.0, 0.5], [0.0, 0.0], 1)
    with pytest.raises(ValueError, match="infeasible"):
        EqualityReduction(p).reduce(p)


def test_primal_compression_is_exact_on_the_null_space():
    plan = EqualityReduction(_p([[1.0, -1.0]], [0.0], [-5.0, -5.0], [5.0, 5.0], [0.0, 0.0], 1))
    np.testing.assert_allclose(plan.compress_primal([2.0, 2.0], check=True), [2.0])
    np.testing.assert_allclose(plan.compress_primal([[1.0, 1.0], [2.0, 2.0]]), [[1.0], [2.0]])
    np.testing.assert_allclose(plan.expand_primal([[1.0], [2.0]]), [[1.0, 1.0], [2.0, 2.0]])
    np.testing.assert_allclose(plan.compress_primal([1.0, 2.0]), [1.5])
    with pytest.raises(ValueError, match="does not satisfy"):
        plan.compress_primal([1.0, 2.0], check=True)


def test_missing_reduced_bound_lifts_but_fails_the_original_dual_gate():
    p = _p([[1.0, -1.0]], [0.0], [-np.inf, -np.inf], [np.inf, np.inf], [1.0, 0.0], 1)
    y = EqualityReduction(p).reduce(p).lift_dual([], [1.0])
    cert = certificate(p, [0.0, 0.0], y)
    assert not cert["certificate_passed"] and cert["dual_violation"] == pytest.approx(1.0)


@pytest.mark.parametrize("value", [True, 0.5, np.nan, np.inf])
def test_scale_ratio_validation(value):
    with pytest.raises(ValueError, match="max_scale_ratio"):
        EqualityReduction(_p([[1.0, -1.0]], [0.0], [0.0, 0.0], [1.0, 1.0], [0.0, 0.0], 1), max_scale_ratio=value)
