"""Exact long-row splitting: the split LP of every real-model fixture has
short rows, the HiGHS optimum of the original maps onto a certified optimum
of the split LP and back, and HiGHS on the split LP reaches the same
objective with a pair that certifies the original LP."""

from pathlib import Path

import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200 import lp_trace
from co_cultivation_metabolic_atlas_b200.rowsplit import RowSplit
from oracle.highs import solve_one

SBML_DIR = Path(__file__).resolve().parent / "golden" / "sbml"


def problems():
    for e in lp_trace.read_manifest(SBML_DIR):
        p, x, y = lp_trace.load_trace_lp(SBML_DIR, e)
        yield e["filename"], p, x, y


@pytest.mark.parametrize("max_length", [64, 24])
def test_split_is_exact_on_real_models(max_length):
    for name, p, x, y in problems():
        plan = RowSplit(p[0], p[5], max_length=max_length)
        sp = plan.split_problem(p)
        lengths = np.diff(sp[0].indptr)
        assert lengths.max() <= max_length + plan.n_aux  # tails hold their z terms
        long_rows = np.diff(p[0].tocsr().indptr) > max_length
        assert plan.active == bool(long_rows.any())
        for r in np.flatnonzero(long_rows):
            pieces = -(-int(np.diff(p[0].tocsr().indptr)[r]) // max_length)
            assert lengths[plan.row_map[r]] <= max_length + pieces - 1
        # the original optimum, extended, certifies the split LP ...
        xs, ys = plan.extend_primal(x), plan.extend_dual(y)
        cert = lp_trace.certificate(sp, xs, ys)
        assert cert["certificate_passed"], (name, cert)
        # ... and restricts back to itself
        xr, yr = plan.restrict(xs, ys)
        np.testing.assert_array_equal(xr, x)
        np.testing.assert_array_equal(yr, y)
        # HiGHS on the split LP: same objective, certified original pair
        st, fun, x2, y2 = solve_one(sp[0], sp[2], sp[3], sp[4], sp[1], sp[5])
        assert st == 0
        assert fun == pytest.approx(float(p[4] @ x), rel=1e-9, abs=1e-9)
        xo, yo = plan.restrict(x2, y2)
        assert lp_trace.certificate(p, xo, yo)["certificate_passed"], name


def test_split_with_inequality_rows_and_batches():
    """A long inequality row keeps its sense and right-hand side after the
    equality block grows by its segment rows; batched (2-D) vectors extend
    row by row."""
    rng = np.random.default_rng(0)
    from scipy.sparse import random as sprandom, vstack, csr_matrix
    eq = sprandom(6, 300, density=0.02, random_state=1, format="csr")
    ub = csr_matrix(rng.uniform(0.1, 1.0, (2, 300)))              # two dense inequality rows
    a = vstack([eq, ub], format="csr")
    plan = RowSplit(a, 6, max_length=64)
    assert plan.n_aux == 2 * 4 and plan.neq == 6 + 8
    assert list(plan.row_map[6:]) == [14, 15]
    rhs = np.concatenate([np.zeros(6), [5.0, 7.0]])
    sp = plan.split_problem((a, rhs, np.zeros(300), np.ones(300), -np.ones(300), 6))
    assert sp[1][14] == 5.0 and sp[1][15] == 7.0 and sp[5] == 14
    X = rng.uniform(0, 1, (3, 300))
    XS = plan.extend_primal(X)
    assert XS.shape == (3, 308)
    act = (sp[0] @ XS.T).T
    np.testing.assert_allclose(act[:, 6:14], 0.0, atol=1e-12)
    np.testing.assert_allclose(act[:, 14:], (ub @ X.T).T, rtol=1e-12)
