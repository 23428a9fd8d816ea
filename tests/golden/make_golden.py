"""Generate the golden fixtures in this directory (run in a container where
the reference checkout is available; the fixtures are committed and the
tests never read the reference at run time).

Fixtures
--------
problem_golden.npz      outputs of the reference's ``_problem``
                        (``src/cpu_repeated_lp.py:119-147``) for a set of
                        ``linprog`` requests, plus the message of each request
                        it rejects.
certificate_golden.npz  outputs of the reference's ``_certificate``
                        (``src/cpu_repeated_lp.py:150-178``) for HiGHS and
                        perturbed primal/dual pairs.
highs_single.npz        HiGHS (SciPy) optima of seeded single-species FBA
                        instances (1,200 x 2,600 generator, first instances).
highs_community.npz     HiGHS optima of seeded three-species instances.

Usage:  python tests/golden/make_golden.py /path/to/reference
"""

from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
from scipy.sparse import csr_matrix

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from tests.golden._reference import reference_root  # noqa: E402
from co_cultivation_metabolic_atlas_b200 import synthetic as syn  # noqa: E402
from oracle import highs  # noqa: E402


def _requests():
    rng = np.random.default_rng(5)
    dense = rng.normal(size=(3, 4))
    dense[0, 1] = 0.0
    dup = csr_matrix((np.array([1.0, 2.0, -1.0, 0.0]), np.array([0, 0, 2, 3]), np.array([0, 2, 4])),
                     shape=(2, 4))
    reqs = [
        ("dense_eq_bounds_pairs", np.array([1.0, -2.0, 0.5, 0.0]),
         dict(A_eq=dense, b_eq=np.array([1.0, 0.0, -2.0]), bounds=[(0, 1), (None, 3), (-1, None), (None, None)])),
        ("eq_and_ub_single_pair", np.array([0.0, 1.0, 0.0, -1.0]),
         dict(A_eq=dense[:1], b_eq=np.array([0.5]), A_ub=dense[1:], b_ub=np.array([1.0, 2.0]), bounds=(0, 10))),
        ("duplicates_and_zeros", np.array([1.0, 1.0, 1.0, 1.0]),
         dict(A_ub=dup, b_ub=np.array([3.0, 4.0]), bounds=np.array([[0, 1]] * 4, dtype=float))),
        ("no_bounds", np.array([-1.0, 0.0, 0.0, 2.0]),
         dict(A_eq=dense, b_eq=np.zeros(3), method='highs')),
        ("object_bounds", np.array([1.0, 2.0, 3.0, 4.0]),
         dict(A_ub=dense[:2], b_ub=np.array([1.0, 1.0]), bounds=np.array([(0, None), (None, 1), (2, 5), (None, None)], dtype=object))),
    ]
    bad = [
        ("nonfinite_objective", np.array([np.nan, 1.0]), dict()),
        ("two_d_objective", np.ones((2, 2)), dict()),
        ("bad_method", np.ones(2), dict(method='interior-point')),
        ("integrality", np.ones(2), dict(integrality=[1, 0])),
        ("rhs_shape", np.ones(2), dict(A_eq=np.ones((1, 2)), b_eq=np.ones(2))),
        ("nonfinite_matrix", np.ones(2), dict(A_eq=np.array([[np.inf, 1.0]]), b_eq=np.ones(1))),
        ("matrix_columns", np.ones(2), dict(A_ub=np.ones((1, 3)), b_ub=np.ones(1))),
        ("lower_gt_upper", np.ones(2), dict(bounds=[(1, 0), (0, 1)])),
        ("nan_bound", np.ones(2), dict(bounds=[(np.nan, 1), (0, 1)])),
        ("bounds_shape", np.ones(3), dict(bounds=[(0, 1), (0, 1)])),
    ]
    return reqs, bad


def problem_golden(ref):
    from src.cpu_repeated_lp import _problem
    reqs, bad = _requests()
    out = {}
    meta = dict(ok=[], bad={})
    for name, c, kw in reqs:
        a, rhs, lo, up, cc, neq = _problem(c, kw)
        meta["ok"].append(name)
        out[f"{name}__c_in"] = c
        out[f"{name}__a_data"] = a.data
        out[f"{name}__a_indices"] = a.indices
        out[f"{name}__a_indptr"] = a.indptr
        out[f"{name}__a_shape"] = np.array(a.shape)
        out[f"{name}__rhs"] = rhs
        out[f"{name}__lower"] = lo
        out[f"{name}__upper"] = up
        out[f"{name}__c"] = cc
        out[f"{name}__neq"] = np.array(neq)
    for name, c, kw in bad:
        try:
            _problem(c, kw)
            meta["bad"][name] = None
        except ValueError as e:
            meta["bad"][name] = str(e)
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(HERE / "problem_golden.npz", **out)


def certificate_golden(ref):
    from src.cpu_repeated_lp import _certificate
    model, lower, upper = syn.single_species_workload(4, m=120, n=260)
    S = model.S
    out = {}
    rows = []
    rng = np.random.default_rng(11)
    for i in range(4):
        st, f, x, y = highs.solve_one(S, lower[i], upper[i], model.cost)
        assert st == 0
        cases = [("highs", x, y), ("x_perturbed", x + rng.normal(scale=1e-4, size=x.shape), y),
                 ("y_perturbed", x, y + rng.normal(scale=1e-3, size=y.shape)),
                 ("zero", np.zeros_like(x), np.zeros_like(y))]
        for name, xx, yy in cases:
            sol = SimpleNamespace(col_value=xx, row_dual=yy, col_dual=model.cost - S.T @ yy,
                                  value_valid=True, dual_valid=True)
            cert = _certificate(S, np.zeros(S.shape[0]), lower[i], upper[i], model.cost, S.shape[0], sol)
            key = f"{i}_{name}"
            out[f"{key}__x"] = xx
            out[f"{key}__y"] = yy
            rows.append(dict(key=key, instance=i, **{k: (float(v) if not isinstance(v, bool) else v)
                                                     for k, v in cert.items()}))
    # an inequality-row case with y_ub sign conventions
    a = csr_matrix(np.array([[1.0, 1.0], [1.0, -1.0], [-1.0, 2.0]]))
    rhs = np.array([1.0, 0.5, 2.0])
    lo = np.array([0.0, -np.inf])
    up = np.array([np.inf, 3.0])
    c = np.array([-1.0, -0.5])
    for name, xx, yy in (("ineq_a", np.array([0.75, 0.25]), np.array([0.0, -0.75, -0.25])),
                         ("ineq_b", np.array([0.5, 0.5]), np.array([-0.6, 0.1, 0.0]))):
        sol = SimpleNamespace(col_value=xx, row_dual=yy, col_dual=c - a.T @ yy, value_valid=True, dual_valid=True)
        cert = _certificate(a, rhs, lo, up, c, 1, sol)
        out[f"{name}__x"] = xx
        out[f"{name}__y"] = yy
        rows.append(dict(key=name, instance=-1, **{k: (float(v) if not isinstance(v, bool) else v)
                                                   for k, v in cert.items()}))
    out["rows"] = np.array(json.dumps(rows))
    np.savez_compressed(HERE / "certificate_golden.npz", **out)


def input_digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def highs_single():
    count = 8
    model, lower, upper = syn.single_species_workload(count)
    res, _ = highs.solve_batch([model.S] * count, lower, upper, [model.cost] * count, workers=8)
    np.savez_compressed(
        HERE / "highs_single.npz",
        fun=np.array([r[1] for r in res]), x=np.stack([r[2] for r in res]),
        y=np.stack([r[3] for r in res]), exchange_lower=lower[:, :model.n_exchange],
        digest=np.array(input_digest(model.S.data, model.S.indices, model.S.indptr, lower, upper)))


def community_bounds(models, medium, biomass, dt=0.05):
    """Exchange lower bounds of every species from a medium state (the same
    Michaelis-Menten rule as the dFBA oracle)."""
    from oracle import dfba
    return [dfba.uptake_lower_bounds(mdl, medium, biomass, dt) for mdl in models]


def highs_community():
    from oracle import dfba
    models = syn.community_models()
    medium, biomass = syn.initial_environments(4)
    out = {}
    for k, mdl in enumerate(models):
        lo = dfba.uptake_lower_bounds(mdl, medium, biomass, 0.05)
        up = np.repeat(mdl.upper[None, :], len(lo), axis=0)
        res, _ = highs.solve_batch([mdl.S] * len(lo), lo, up, [mdl.cost] * len(lo), workers=8)
        out[f"s{k}_fun"] = np.array([r[1] for r in res])
        out[f"s{k}_x"] = np.stack([r[2] for r in res])
        out[f"s{k}_digest"] = np.array(input_digest(mdl.S.data, mdl.S.indices, lo, up))
    np.savez_compressed(HERE / "highs_community.npz", **out)


if __name__ == "__main__":
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else reference_root())
    sys.path.insert(0, str(ref))
    problem_golden(ref)
    certificate_golden(ref)
    highs_single()
    highs_community()
    print("golden fixtures written to", HERE)
