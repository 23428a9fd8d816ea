"""SBML reader: known answers from the reference's own tests on its
consortium models (read when the reference checkout is named by the
``FBALP_REFERENCE`` environment variable), and the committed real-model LP
fixtures (always)."""

import json
import os
from pathlib import Path

import numpy as np
import pytest
from scipy.optimize import linprog

from co_cultivation_metabolic_atlas_b200 import lp_trace, sbml

REFERENCE = Path(os.environ.get("FBALP_REFERENCE", "")) if os.environ.get("FBALP_REFERENCE") else None
SBML_DIR = Path(__file__).resolve().parent / "golden" / "sbml"
needs_reference = pytest.mark.skipif(REFERENCE is None or not (REFERENCE / "models" / "sbml").is_dir(),
                                     reason="reference models not present (set FBALP_REFERENCE)")


def _open_growth(m):
    """``_fully_open_growth`` of ``tests/test_wcfs1_2022_repair.py:13-19``:
    every exchange at ``lower <= -20``, ``upper >= 1000``, maximise the
    objective."""
    lo, up = m.lower.copy(), m.upper.copy()
    lo[m.exchanges] = np.minimum(lo[m.exchanges], -20.0)
    up[m.exchanges] = np.maximum(up[m.exchanges], 1000.0)
    r = linprog(m.fba_cost(), A_eq=m.S, b_eq=np.zeros(m.S.shape[0]), bounds=np.column_stack([lo, up]),
                method="highs")
    return -r.fun if r.status == 0 else 0.0


@needs_reference
def test_wcfs1_repaired_model_pins():
    """``tests/test_wcfs1_2022_repair.py``: model id, biomass coefficients,
    no peptido_LPL_c in the repaired biomass, positive open growth; the
    deposited model's biomass holds peptido_LPL_c and cannot grow."""
    m = sbml.read_sbml(REFERENCE / "models/sbml/final_consortium/Lactobacillus_plantarum.xml")
    assert m.id == "WCFS1_Koduru2022_repaired"
    coef = m.reaction_stoichiometry("biomass")
    assert coef["PGlac2_c"] == pytest.approx(-0.1462)
    assert coef["CPS_LPL2_c"] == pytest.approx(-0.1294)
    assert coef["nad_c"] == pytest.approx(-0.002)
    assert "peptido_LPL_c" not in coef
    assert "UGMDDS2" in m.reactions
    assert _open_growth(m) > 1e-6
    src = sbml.read_sbml(REFERENCE / "models/sbml/reference/Lactiplantibacillus_plantarum_WCFS1_Koduru2022.xml")
    assert "peptido_LPL_c" in src.reaction_stoichiometry("biomass")
    assert "UGMDDS2" not in src.reactions
    assert _open_growth(src) == pytest.approx(0.0, abs=1e-9)
    assert len(m.exchanges) == len(src.exchanges)
    assert len(m.reactions) == len(src.reactions) + 1


@needs_reference
def test_consortium_model_pins():
    """``tests/test_science_integrity.py``: NS21's PHA unit is cytosolic
    (compartment ``C_c``); OR16 has no ODTD metabolite and its Lcp reaction
    ``R_LCP`` is closed; the plantarum model with every exchange at -10
    solves and secretes no biosurfactant."""
    base = REFERENCE / "models/sbml/final_consortium"
    ns21 = sbml.read_sbml(base / "Rhizobacter_gummiphilus_NS21.xml")
    assert ns21.compartments[ns21.metabolite_index("pha_c")] == "C_c"
    or16 = sbml.read_sbml(base / "Actinoplanes_sp_OR16_lcp.xml")
    assert not [x for x in or16.metabolites if "odtd" in x.lower()]
    j = or16.reaction_index("R_LCP")
    assert (or16.lower[j], or16.upper[j]) == (0.0, 0.0)
    lp = sbml.read_sbml(base / "Lactobacillus_plantarum.xml")
    lo = lp.lower.copy()
    lo[lp.exchanges] = -10.0
    r = linprog(lp.fba_cost(), A_eq=lp.S, b_eq=np.zeros(lp.S.shape[0]), bounds=np.column_stack([lo, lp.upper]),
                method="highs")
    assert r.status == 0
    if "EX_biosurfactant_e" in lp.reactions:
        assert abs(r.x[lp.reaction_index("EX_biosurfactant_e")]) < 1e-12


@needs_reference
def test_reader_on_every_consortium_model():
    """Every model parses with one objective column, an external
    compartment and exchange reactions that each touch one external
    metabolite; the committed fixtures hold exactly these matrices."""
    meta = json.loads((SBML_DIR / "models.json").read_text())
    for key, info in meta.items():
        m = sbml.read_sbml(REFERENCE / info["source"])
        assert (m.S.shape, m.S.nnz) == ((info["rows"], info["columns"]), info["nonzeros"])
        assert list(m.exchanges) == info["exchanges"]
        assert int(np.flatnonzero(m.objective)[0]) == info["objective_column"]
        for j in m.exchanges[:20]:
            assert m.compartments[m.metabolite_index(m.exchange_metabolite(j))] == m.external_compartment


def test_sbml_fixtures_load_and_certify():
    """The real-model LPs load through the trace loader (checksums, hashes,
    certificate of the recorded HiGHS pair) and their objectives are the
    recorded HiGHS optima."""
    meta = json.loads((SBML_DIR / "models.json").read_text())
    entries = lp_trace.read_manifest(SBML_DIR)
    assert len(entries) == 2 * len(meta)
    for e in entries:
        problem, x, y = lp_trace.load_trace_lp(SBML_DIR, e)
        key, variant = e["filename"][:-4].rsplit("_", 1)
        assert float(problem[4] @ x) == pytest.approx(meta[key]["highs_objective"][variant], rel=1e-12)


FBC2 = """<?xml version="1.0" encoding="UTF-8"?>
<sbml xmlns="http://www.sbml.org/sbml/level3/version1/core"
      xmlns:fbc="http://www.sbml.org/sbml/level3/version1/fbc/version2" level="3" version="1" fbc:required="false">
  <model id="toy" name="toy model" fbc:strict="true">
    <listOfCompartments>
      <compartment id="C_c" name="cytosol" constant="true"/>
      <compartment id="C_x" name="extracellular space" constant="true"/>
    </listOfCompartments>
    <listOfSpecies>
      <species id="M_a_c" compartment="C_c" boundaryCondition="false" hasOnlySubstanceUnits="false" constant="false"/>
      <species id="M_a_x" compartment="C_x" boundaryCondition="false" hasOnlySubstanceUnits="false" constant="false"/>
      <species id="M_b_c" compartment="C_c" boundaryCondition="false" hasOnlySubstanceUnits="false" constant="false"/>
      <species id="M_src" compartment="C_x" boundaryCondition="true" hasOnlySubstanceUnits="false" constant="false"/>
    </listOfSpecies>
    <listOfParameters>
      <parameter id="lo" value="-INF" constant="true"/>
      <parameter id="up" value="INF" constant="true"/>
      <parameter id="zero" value="0" constant="true"/>
      <parameter id="ten" value="10" constant="true"/>
    </listOfParameters>
    <listOfReactions>
      <reaction id="R_EX_a" reversible="true" fbc:lowerFluxBound="lo" fbc:upperFluxBound="ten">
        <listOfReactants><speciesReference species="M_a_x" stoichiometry="1" constant="true"/></listOfReactants>
      </reaction>
      <reaction id="R_T_a" reversible="false" fbc:lowerFluxBound="zero" fbc:upperFluxBound="up">
        <listOfReactants><speciesReference species="M_a_x" stoichiometry="1" constant="true"/></listOfReactants>
        <listOfProducts><speciesReference species="M_a_c" stoichiometry="1" constant="true"/></listOfProducts>
      </reaction>
      <reaction id="R_CONV" reversible="true">
        <listOfReactants><speciesReference species="M_a_c" stoichiometry="2" constant="true"/>
                         <speciesReference species="M_src" stoichiometry="1" constant="true"/></listOfReactants>
        <listOfProducts><speciesReference species="M_b_c" stoichiometry="1" constant="true"/>
                        <speciesReference species="M_a_c" stoichiometry="0.5" constant="true"/></listOfProducts>
      </reaction>
      <reaction id="R_SINK_b" reversible="false">
        <listOfReactants><speciesReference species="M_b_c" stoichiometry="1" constant="true"/></listOfReactants>
      </reaction>
    </listOfReactions>
    <fbc:listOfObjectives fbc:activeObjective="o2">
      <fbc:objective fbc:id="o1" fbc:type="maximize">
        <fbc:listOfFluxObjectives><fbc:fluxObjective fbc:reaction="R_SINK_b" fbc:coefficient="1"/></fbc:listOfFluxObjectives>
      </fbc:objective>
      <fbc:objective fbc:id="o2" fbc:type="minimize">
        <fbc:listOfFluxObjectives><fbc:fluxObjective fbc:reaction="R_T_a" fbc:coefficient="2"/></fbc:listOfFluxObjectives>
      </fbc:objective>
    </fbc:listOfObjectives>
  </model>
</sbml>
"""


def test_reader_format_rules(tmp_path):
    """COBRA's id rules (one R_ / M_ prefix removed, compartments kept),
    boundary species without rows, accumulated stoichiometry of a species on
    both sides, INF bounds, default bounds by reversibility, the active
    (minimised) objective, and the external compartment found by name."""
    path = tmp_path / "toy.xml"
    path.write_text(FBC2)
    m = sbml.read_sbml(path)
    assert m.id == "toy" and m.reactions == ["EX_a", "T_a", "CONV", "SINK_b"]
    assert m.metabolites == ["a_c", "a_x", "b_c"] and m.compartments == ["C_c", "C_x", "C_c"]
    A = m.S.toarray()
    np.testing.assert_array_equal(A[:, 2], [-1.5, 0.0, 1.0])       # a_c: -2 + 0.5; M_src dropped
    np.testing.assert_array_equal(A[:, 0], [0.0, -1.0, 0.0])
    assert m.lower.tolist() == [-np.inf, 0.0, -1000.0, 0.0]
    assert m.upper.tolist() == [10.0, np.inf, 1000.0, 1000.0]
    assert m.direction == "min" and m.objective.tolist() == [0.0, 2.0, 0.0, 0.0]
    np.testing.assert_array_equal(m.fba_cost(), m.objective)
    assert m.external_compartment == "C_x" and m.exchanges.tolist() == [0]
    assert m.exchange_metabolite(0) == "a_x"


def test_reader_fbc_version_1_bounds(tmp_path):
    """FBC version 1 keeps flux bounds in a listOfFluxBounds."""
    text = FBC2.replace("fbc/version2", "fbc/version1")
    for name in ("lo", "up", "zero", "ten"):
        text = text.replace(f' fbc:lowerFluxBound="{name}"', "").replace(f' fbc:upperFluxBound="{name}"', "")
    text = text.replace("    <fbc:listOfObjectives", """    <fbc:listOfFluxBounds>
      <fbc:fluxBound fbc:reaction="R_EX_a" fbc:operation="greaterEqual" fbc:value="-5"/>
      <fbc:fluxBound fbc:reaction="R_EX_a" fbc:operation="lessEqual" fbc:value="7"/>
      <fbc:fluxBound fbc:reaction="R_CONV" fbc:operation="equal" fbc:value="2"/>
    </fbc:listOfFluxBounds>
    <fbc:listOfObjectives""")
    path = tmp_path / "toy1.xml"
    path.write_text(text)
    m = sbml.read_sbml(path)
    assert m.lower.tolist() == [-5.0, 0.0, 2.0, 0.0]
    assert m.upper.tolist() == [7.0, 1000.0, 2.0, 1000.0]


@pytest.mark.parametrize("edit,match", [
    (('fbc:upperFluxBound="ten"', 'fbc:upperFluxBound="eleven"'), "undefined bound parameter eleven"),
    (('fbc:lowerFluxBound="zero" fbc:upperFluxBound="up"', 'fbc:lowerFluxBound="ten" fbc:upperFluxBound="zero"'),
     "above upper bound"),
])
def test_reader_rejects_inconsistent_bounds(tmp_path, edit, match):
    path = tmp_path / "bad.xml"
    path.write_text(FBC2.replace(*edit))
    with pytest.raises(ValueError, match=match):
        sbml.read_sbml(path)
