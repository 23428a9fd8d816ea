"""Generate the real-model LP fixtures in ``sbml/`` from the reference's
consortium SBML files, read with this package's SBML reader.  Run in a
container where the reference checkout is available; the fixtures are
committed and the tests never read the reference.

For each model two FBA LPs (``S v = 0``, maximise the model's objective)
are written in the reference's LP-trace format (``src/lp_trace.py:43-57``)
with their HiGHS primal/dual pair:

* ``default``: the SBML bounds clipped to [-1000, 1000], as the reference
  simulator clips them before solving (``src/dfba_simulator.py:575-577``);
* ``open``: additionally every exchange opened to ``lower <= -20,
  upper >= 1000`` (the fully-open medium of
  ``tests/test_wcfs1_2022_repair.py:13-19``).

``sbml/models.json`` records, per model, its id, dimensions, exchange
columns and objective column, for the batched tests.

Usage:  python tests/golden/make_sbml_traces.py /path/to/reference
"""

from __future__ import annotations

import json
import shutil
import sys
from pathlib import Path

import numpy as np
from scipy.optimize import linprog

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from tests.golden._reference import reference_root  # noqa: E402
from co_cultivation_metabolic_atlas_b200 import lp_trace, sbml  # noqa: E402

MODELS = {
    "lactobacillus_plantarum": "models/sbml/final_consortium/Lactobacillus_plantarum.xml",
    "rhizobacter_gummiphilus_ns21": "models/sbml/final_consortium/Rhizobacter_gummiphilus_NS21.xml",
    "actinoplanes_or16": "models/sbml/final_consortium/Actinoplanes_sp_OR16_lcp.xml",
    "bacillus_subtilis_iyo844": "models/sbml/helper_candidates/Bacillus_subtilis_168_iYO844_curated.xml",
    "propionibacterium_shermanii": "models/sbml/helper_candidates/Propionibacterium_freudenreichii_shermanii_curated.xml",
}


def highs(a, lower, upper, c):
    res = linprog(c, A_eq=a, b_eq=np.zeros(a.shape[0]), bounds=np.column_stack([lower, upper]), method="highs-ds",
                  options=dict(presolve=True, primal_feasibility_tolerance=1e-10,
                               dual_feasibility_tolerance=1e-10))
    if res.status != 0:
        raise RuntimeError(res.message)
    return np.asarray(res.x), np.asarray(res.eqlin.marginals)


def main(reference):
    out = HERE / "sbml"
    if out.exists():
        shutil.rmtree(out)
    out.mkdir()
    entries, meta = [], {}
    for key, rel in MODELS.items():
        m = sbml.read_sbml(Path(reference) / rel)
        lower = np.clip(m.lower, -1000.0, 1000.0)
        upper = np.clip(m.upper, -1000.0, 1000.0)
        c = m.fba_cost()
        a = m.S.tocsr()
        variants = {"default": (lower, upper)}
        lo, up = lower.copy(), upper.copy()
        lo[m.exchanges] = np.minimum(lo[m.exchanges], -20.0)
        up[m.exchanges] = np.maximum(up[m.exchanges], 1000.0)
        variants["open"] = (lo, up)
        objectives = {}
        for name, (l, u) in variants.items():
            x, y = highs(a, l, u, c)
            problem = (a, np.zeros(a.shape[0]), l, u, c, a.shape[0])
            entries.append(lp_trace.write_trace_lp(out / f"{key}_{name}.npz", problem, reference_x=x,
                                                   reference_y=y))
            objectives[name] = float(c @ x)
        meta[key] = dict(id=m.id, source=rel, rows=a.shape[0], columns=a.shape[1], nonzeros=int(a.nnz),
                         exchanges=[int(j) for j in m.exchanges],
                         objective_column=int(np.flatnonzero(m.objective)[0]),
                         highs_objective=objectives)
        print(key, a.shape, a.nnz, objectives)
    lp_trace.write_manifest(out, entries)
    (out / "models.json").write_text(json.dumps(meta, indent=1, sort_keys=True))
    # the committed files must load and certify through the package loader
    for e in lp_trace.read_manifest(out):
        lp_trace.load_trace_lp(out, e)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else reference_root())
