"""Request normalisation matches the reference's ``_problem`` on golden
vectors produced by the reference itself (tests/golden/make_golden.py)."""
import json

import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200.problem import normalize, request
from tests.golden.make_golden import _requests


@pytest.fixture(scope="module")
def golden(golden_dir):
    return np.load(golden_dir / "problem_golden.npz", allow_pickle=False)


def test_normalized_problems_match_reference(golden):
    meta = json.loads(str(golden["meta"]))
    reqs, _ = _requests()
    assert [r[0] for r in reqs] == meta["ok"]
    for name, c, kw in reqs:
        a, rhs, lo, up, cc, neq = normalize(c, kw)
        np.testing.assert_array_equal(golden[f"{name}__c_in"], c)
        np.testing.assert_array_equal(a.data, golden[f"{name}__a_data"])
        np.testing.assert_array_equal(a.indices, golden[f"{name}__a_indices"])
        np.testing.assert_array_equal(a.indptr, golden[f"{name}__a_indptr"])
        assert tuple(a.shape) == tuple(golden[f"{name}__a_shape"])
        np.testing.assert_array_equal(rhs, golden[f"{name}__rhs"])
        np.testing.assert_array_equal(lo, golden[f"{name}__lower"])
        np.testing.assert_array_equal(up, golden[f"{name}__upper"])
        np.testing.assert_array_equal(cc, golden[f"{name}__c"])
        assert neq == int(golden[f"{name}__neq"])


# The two messages that name the reference's CPU comparator are reworded;
# every other rejection carries the reference's message verbatim.
REWORDED = {"bad_method", "integrality"}


def test_rejections_match_reference(golden):
    meta = json.loads(str(golden["meta"]))
    _, bad = _requests()
    for name, c, kw in bad:
        expected = meta["bad"][name]
        assert expected is not None
        with pytest.raises(ValueError) as info:
            normalize(c, kw)
        if name not in REWORDED:
            assert str(info.value) == expected


def test_request_round_trip(golden):
    reqs, _ = _requests()
    for name, c, kw in reqs:
        p = normalize(c, kw)
        q = normalize(*request(p))
        for u, v in zip(p[1:5], q[1:5]):
            np.testing.assert_array_equal(u, v)
        assert (p[0] != q[0]).nnz == 0 and p[5] == q[5]


def test_normalize_batch_shares_one_objective_copy_per_object():
    """Requests that pass the same objective object share one validated
    copy; it does not follow later changes to the caller's array, and a
    non-finite objective is still rejected."""
    from co_cultivation_metabolic_atlas_b200.problem import normalize_batch
    c = np.array([1.0, -2.0, 0.5])
    a = np.array([[1.0, 1.0, 0.0]])
    kw = dict(A_eq=a, b_eq=np.zeros(1), bounds=[(0, 1)] * 3)
    out = normalize_batch([(c, kw), (c, dict(kw)), (c.copy(), dict(kw))])
    assert out[0][4] is out[1][4] and out[2][4] is not out[0][4]
    c[0] = 7.0
    np.testing.assert_array_equal(out[0][4], [1.0, -2.0, 0.5])
    np.testing.assert_array_equal(out[2][4], [1.0, -2.0, 0.5])
    bad = np.array([1.0, np.inf, 0.0])
    with pytest.raises(ValueError):
        normalize_batch([(bad, kw), (bad, dict(kw))])
