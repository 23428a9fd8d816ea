"""Generate the LP-trace fixtures in ``traces/`` with the REFERENCE's own
trace writer (``src/lp_trace.py:43-57``), so the engine's loader is tested on
files and manifest entries the reference produced.  Run in a container where
the reference checkout is available; the fixtures are committed and the tests
never read the reference.

Three seeded FBA LPs (a small synthetic species and a one-inequality variant)
are solved with HiGHS (SciPy) and written with their HiGHS primal/dual pair;
one entry carries step/stage/environment labels.  The reference's loader is
run on the result here as a check.  ``trace_hashes.json`` records the
reference's ``problem_hash`` of the normalised requests of
``problem_golden.npz``'s cases built below.

Usage:  python tests/golden/make_traces.py /path/to/reference
"""

from __future__ import annotations

import json
import shutil
import sys
from pathlib import Path

import numpy as np
from scipy.sparse import csr_matrix, vstack

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from tests.golden._reference import reference_root  # noqa: E402
from co_cultivation_metabolic_atlas_b200 import synthetic as syn  # noqa: E402
from oracle import highs  # noqa: E402


def problems():
    model, lower, upper = syn.single_species_workload(3, m=120, n=260, seed=3)
    out = []
    for i in range(2):
        a = csr_matrix(model.S)
        out.append((a, np.zeros(a.shape[0]), lower[i], upper[i], model.cost.copy(), a.shape[0]))
    # a variant with one inequality row (sum of the first five fluxes <= 7)
    a = csr_matrix(model.S)
    row = np.zeros((1, a.shape[1]))
    row[0, :5] = 1.0
    a2 = vstack([a, csr_matrix(row)], format="csr")
    out.append((a2, np.concatenate([np.zeros(a.shape[0]), [7.0]]), lower[2], upper[2], model.cost.copy(),
                a.shape[0]))
    return out


def main():
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else reference_root())
    sys.path.insert(0, str(ref))
    from src.cpu_repeated_lp import _problem
    from src.lp_trace import load_trace_lp, problem_hash, problem_request, write_trace_lp
    out = HERE / "traces"
    if out.exists():
        shutil.rmtree(out)
    out.mkdir()
    entries = []
    names = ["lp_a.npz", "lp_b.npz", "lp_001_2_004.npz"]
    for k, prob in enumerate(problems()):
        p = _problem(*problem_request(prob))
        a, rhs, lower, upper, c, neq = p
        st, fun, x, y = highs.solve_one(a, lower, upper, c, rhs=rhs, neq=neq)
        assert st == 0
        entry = write_trace_lp(out / names[k], p, reference_x=x, reference_y=y)
        if k == 2:
            entry.update(step=1, stage="exchange", environment_id=4)
        entries.append(entry)
    (out / "manifest.json").write_text(json.dumps({"traces": entries}, indent=1, sort_keys=True))
    for e in entries:  # the reference's own loader accepts what it wrote
        load_trace_lp(out, e)
    hashes = {}
    for k, prob in enumerate(problems()):
        hashes[names[k]] = problem_hash(_problem(*problem_request(prob)))
    (HERE / "trace_hashes.json").write_text(json.dumps(hashes, indent=1, sort_keys=True))
    print(f"wrote {len(entries)} traces and {len(hashes)} hashes")


if __name__ == "__main__":
    main()
