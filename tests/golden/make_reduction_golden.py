"""Generate ``reduction_golden.npz``: outputs of the reference's
``HomogeneousEqualityReduction`` (``src/lp_equality_reduction.py``) on seeded
LPs, for the parity tests of ``co_cultivation_metabolic_atlas_b200.reduction``.
Run in a container where the reference checkout is available; the fixture
is committed and the tests never read the reference.

Cases: the three community species (default bounds, biomass objective) and
a seeded LP with chains, a scaled relation, a cycle and negative weights.
For each: the plan (transform, rows, representatives, dual lift map), the
reduced problem, the witnesses, and the lifted duals of a seeded reduced
dual vector (with its consistent reduced cost).

Usage:  python tests/golden/make_reduction_golden.py /path/to/reference
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
from scipy.sparse import csr_matrix

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from tests.golden._reference import reference_root  # noqa: E402
from co_cultivation_metabolic_atlas_b200 import synthetic as syn  # noqa: E402


def cases():
    out = {}
    for k, mdl in enumerate(syn.community_models(seed=0)):
        out[f"species{k}"] = (mdl.S, np.zeros(mdl.S.shape[0]), mdl.lower, mdl.upper, mdl.cost, mdl.S.shape[0])
    rng = np.random.default_rng(17)
    n, m = 40, 30
    dense = np.zeros((m, n))
    for r in range(10):                       # chains and a cycle of two-entry rows
        p, q = r, r + 1
        dense[r, p], dense[r, q] = rng.choice([1.0, 2.0, -0.5]), -rng.choice([1.0, 3.0, 0.25])
    dense[10, 0], dense[10, 5] = 1.0, -1.0    # closes a cycle (kept)
    dense[11, 20], dense[11, 21] = 1.0, 1.0   # negative weight pair
    for r in range(12, m):                    # general rows
        cols = rng.choice(n, 5, replace=False)
        dense[r, cols] = rng.normal(size=5)
    neq = 25
    rhs = np.zeros(m)
    rhs[neq:] = rng.uniform(1, 5, m - neq)
    lower = -rng.uniform(0, 10, n)
    upper = rng.uniform(0, 10, n)
    out["chains"] = (csr_matrix(dense), rhs, lower, upper, rng.normal(size=n), neq)
    return out


def main():
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else reference_root())
    sys.path.insert(0, str(ref))
    from src.lp_equality_reduction import HomogeneousEqualityReduction
    blob = {}
    rng = np.random.default_rng(3)
    for name, p in cases().items():
        plan = HomogeneousEqualityReduction(p)
        red = plan.reduce(p)
        t = plan.transform.tocoo()
        dl = plan.dual_lift_map.tocoo()
        ra, rrhs, rlo, rup, rc, rneq = red.problem
        ry = rng.normal(size=len(plan.kept_rows))
        rcost = np.asarray(plan.transform.T @ (p[4] - red.kept_matrix.T @ ry)).ravel()
        y = red.lift_dual(ry, rcost)
        for key, val in dict(t_row=t.row, t_col=t.col, t_val=t.data, eliminated=plan.eliminated_rows,
                             kept=plan.kept_rows, representatives=plan.representatives,
                             dl_row=dl.row, dl_col=dl.col, dl_val=dl.data, ra_indptr=ra.indptr,
                             ra_indices=ra.indices, ra_data=ra.data, ra_shape=ra.shape, rrhs=rrhs, rlo=rlo,
                             rup=rup, rc=rc, rneq=rneq, lower_witness=red.lower_witness,
                             upper_witness=red.upper_witness, ry=ry, rcost=rcost, y=y).items():
            blob[f"{name}__{key}"] = np.asarray(val)
    np.savez_compressed(HERE / "reduction_golden.npz", **blob)
    print("wrote reduction_golden.npz with", len(blob), "arrays")


if __name__ == "__main__":
    main()
