"""The C-ABI library loads, exports every declared symbol, and its host-only
preprocessing matches the oracle -- no GPU needed."""
import ctypes
import re

import numpy as np
import pytest
from scipy.sparse import csr_matrix

from tests.conftest import ROOT


def declared_symbols():
    text = "".join(p.read_text() for p in sorted((ROOT / "include").glob("*.h")))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fbalp_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_symbols()
    for required in ("fbalp_engine_create", "fbalp_engine_set_instances", "fbalp_engine_solve",
                     "fbalp_engine_destroy", "fbalp_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol(native_built):
    lib = ctypes.CDLL(str(native_built))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert missing == []


def test_defaults(native_built):
    from co_cultivation_metabolic_atlas_b200 import _native as N
    o = N.default_options()
    p = N.default_solve_params()
    assert (o.ruiz_iterations, o.power_iterations, o.warps_per_block) == (10, 256, 16)
    assert o.step_safety == pytest.approx(0.99)
    assert p.precision == N.PRECISION_MIXED and p.check_every == 64
    assert p.tol_gap == pytest.approx(1e-7) and p.fp32_tol_gap == pytest.approx(1e-4)
    assert p.fp64_stall_checks == 8 and p.floor_tol == pytest.approx(1e-7)
    # the fields after the original ones: read through the ctypes mirror, so
    # a layout that drifted from the header would read other fields' bytes
    assert p.fp32_recentre == 1 and p.fp32_values_phase == 1
    assert (p.gate_primal, p.gate_dual, p.gate_gap) == pytest.approx((1e-5, 1e-7, 1e-7))
    assert p.primal_weight_smoothing == pytest.approx(0.5)
    assert o.pair_instances == 1 and o.spread_banks == 1


def test_solve_config_converts_and_checks_the_schedule_fields():
    from co_cultivation_metabolic_atlas_b200.engine import EngineOptions, SolveConfig
    for value, want in ((True, 1), (False, 0), (0, 0), (1, 1), (2, 2)):
        assert SolveConfig(fp32_values_phase=value).native().fp32_values_phase == want
    for bad in (3, -1, 1.5, "2"):
        with pytest.raises(ValueError):
            SolveConfig(fp32_values_phase=bad).native()
    q = SolveConfig(gate_primal=2e-5, primal_weight_smoothing=0.3).native()
    assert q.gate_primal == pytest.approx(2e-5) and q.primal_weight_smoothing == pytest.approx(0.3)
    assert EngineOptions(spread_banks=False).native().spread_banks == 0


def test_host_preprocessing_matches_oracle(native_built):
    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    from co_cultivation_metabolic_atlas_b200.engine import prepare_matrix
    from oracle import pdhg
    model, _, _ = syn.single_species_workload(1, m=300, n=650)
    got = prepare_matrix(model.S)
    ref = pdhg.prepare(model.S)
    np.testing.assert_allclose(got["dr"], ref.dr, rtol=1e-14, atol=0)
    np.testing.assert_allclose(got["dc"], ref.dc, rtol=1e-14, atol=0)
    assert got["sigma_max"] == pytest.approx(ref.sigma_max, rel=1e-12)
    assert got["eta"] == pytest.approx(ref.eta, rel=1e-12)
    # Pock-Chambolle scaling bounds the spectral norm by one
    assert got["sigma_max"] <= 1.0 + 1e-12


def test_preprocessing_of_duplicates_equals_summed_matrix(native_built):
    from co_cultivation_metabolic_atlas_b200.engine import prepare_matrix
    dup = csr_matrix((np.array([1.0, 2.0, -1.0, 0.0, 4.0]), np.array([0, 0, 2, 1, 1]),
                      np.array([0, 2, 4, 5])), shape=(3, 3))
    summed = csr_matrix(np.array([[3.0, 0, 0], [0, 0, -1.0], [0, 4.0, 0]]))
    a = prepare_matrix(dup)
    b = prepare_matrix(summed)
    np.testing.assert_array_equal(a["dr"], b["dr"])
    np.testing.assert_array_equal(a["dc"], b["dc"])


@pytest.mark.parametrize("case,match", [
    ("index", "column index out of range"),
    ("nan", "finite"),
    ("ptr", "monotone"),
])
def test_invalid_matrices_are_rejected(native_built, case, match):
    from co_cultivation_metabolic_atlas_b200 import _native as N
    lib = N.load()
    indptr = np.array([0, 2, 3], dtype=np.int64)
    indices = np.array([0, 1, 1], dtype=np.int32)
    values = np.array([1.0, 2.0, 3.0])
    if case == "index":
        indices[2] = 7
    elif case == "nan":
        values[1] = np.nan
    else:
        indptr = np.array([0, 3, 2], dtype=np.int64)
    dr = np.empty(2)
    dc = np.empty(2)
    code = lib.fbalp_prepare_matrix(2, 2, indptr.ctypes.data_as(N.c_int64_p),
                                    indices.ctypes.data_as(N.c_int32_p),
                                    values.ctypes.data_as(N.c_double_p), None,
                                    dr.ctypes.data_as(N.c_double_p), dc.ctypes.data_as(N.c_double_p),
                                    None, None)
    assert code == N.FBALP_ERR_INVALID
    assert match in lib.fbalp_last_error().decode()


def test_engine_entry_points_reject_null_handles(native_built):
    from co_cultivation_metabolic_atlas_b200 import _native as N
    lib = N.load()
    assert lib.fbalp_engine_destroy(None) == N.FBALP_ERR_INVALID
    assert lib.fbalp_engine_set_instances(None, 1, None, None, None, None, None) == N.FBALP_ERR_INVALID
    p = N.default_solve_params()
    assert lib.fbalp_engine_solve(None, None, None, None, ctypes.byref(p), None, None, None, None,
                                  None, None, None) == N.FBALP_ERR_INVALID
    out = ctypes.c_void_p()
    assert lib.fbalp_engine_create(0, None, None, None, None, None, None, None, None,
                                   ctypes.byref(out)) == N.FBALP_ERR_INVALID
    assert out.value is None


def test_scaled_certificate_rejects_invalid_arguments(native_built):
    """Argument checks of the batched certificate run on the host before any
    device call (a zero-instance call with valid arguments is a no-op)."""
    from co_cultivation_metabolic_atlas_b200 import _native as N
    lib = N.load()
    fake = ctypes.c_void_p(16)        # never dereferenced: every call below returns on the host

    def call(count=0, rows=2, cols=3, neq=1, npatch=0, groups=1, prow=fake, pcol=fake, x=fake):
        return lib.fbalp_scaled_certificate(count, rows, cols, neq, fake, fake, fake, fake, fake, fake,
                                            npatch, prow, pcol, None, x, fake, fake, fake, fake, fake,
                                            fake, fake, groups, fake, fake, fake, fake, None)

    assert call() == N.FBALP_OK
    for kwargs, match in [({"neq": 3}, "dimensions"), ({"cols": 0}, "dimensions"), ({"groups": 0}, "dimensions"),
                          ({"count": -1}, "dimensions"), ({"npatch": N.MAX_PATCHES + 1}, "npatch"),
                          ({"npatch": 1, "prow": None}, "npatch"), ({"x": None}, "NULL")]:
        assert call(**kwargs) == N.FBALP_ERR_INVALID, kwargs
        assert match in lib.fbalp_last_error().decode(), kwargs
