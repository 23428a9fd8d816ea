"""The engine on the reference's genome-scale consortium models (fixtures of
their FBA LPs, read by the SBML reader): the ten LPs (five models, default
and fully open media) replayed through the drop-in backend in one uneven
launch, against their HiGHS optima.  Cold solves of these LPs take 0.8-3.1e5
iterations (about 100x the synthetic workload): they finish in the
backend's second GPU pass."""

import shutil
from pathlib import Path

import pytest

from co_cultivation_metabolic_atlas_b200 import lp_trace

pytestmark = pytest.mark.gpu

SBML_DIR = Path(__file__).resolve().parent / "golden" / "sbml"
OBJ_TOL = 1e-6
COLD_CAP = 1_000_000


def test_real_model_traces_replay_through_the_backend(tmp_path, forbid_cpu_optimizers):
    from co_cultivation_metabolic_atlas_b200 import B200LPBackend
    d = tmp_path / "sbml"
    shutil.copytree(SBML_DIR, d)
    # default drop-in settings: the first pass's 20 k cap stops every one of
    # these LPs, the second GPU pass (retry_iterations, 1e6) finishes them
    be = B200LPBackend(mode="cold")
    assert be.split_rows is None and be.retry_iterations == COLD_CAP
    rows, ref = lp_trace.replay(d, be)
    be.close()
    assert len(rows) == 10
    assert be.history[-1]["cpu_lp_calls"] == 0
    for r, fun in zip(rows, ref):
        assert r.success, r.message
        assert abs(r.fun - fun) <= OBJ_TOL * max(1.0, abs(fun)), (r.fun, fun)
    print("iterations", be.history[-1]["iterations"], f"solve {be.history[-1]['solve_seconds']:.1f} s")
