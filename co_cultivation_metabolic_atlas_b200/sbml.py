"""Minimal SBML reader for genome-scale flux-balance models (no COBRA).

The reference loads its consortium models with ``cobra.io.read_sbml_model``
and turns each into ``S v = 0, l <= v <= u, max c.v``
(``create_stoichiometric_matrix``, ``src/dfba_simulator.py:1061-1102``;
``src/community_solver.py:770-790``).  This reader extracts exactly the parts
of an SBML Level 3 file with the FBC package (versions 1 and 2) that the LP
path needs:

* species -> metabolites (rows, in document order), their compartments;
* reactions -> columns (document order) with the stoichiometry of their
  reactants (negative) and products (positive); a species listed twice in a
  reaction accumulates, as COBRA does;
* flux bounds from ``fbc:lowerFluxBound`` / ``fbc:upperFluxBound`` parameter
  references (FBC v2) or ``fbc:listOfFluxBounds`` (FBC v1); ``INF`` values
  become infinities; a reaction without a bound gets ``[-1000, 1000]``
  (``[0, 1000]`` if irreversible), COBRA's defaults; a reference to an
  undefined parameter, or a lower bound above the upper one, is an error
  (COBRA refuses both);
* the active objective (``fbc:listOfObjectives``): coefficients and
  direction.

Identifiers follow COBRA's default SBML id handling: one leading ``R_`` is
removed from reaction ids and one leading ``M_`` from species ids;
compartment ids are kept.  Boundary species (``boundaryCondition="true"``)
are not metabolites (no row).  Exchange reactions are COBRA's
``model.exchanges``: reactions with exactly one metabolite, in the external
compartment (a compartment whose id is ``e`` / ``C_e`` or whose name says
extracellular, otherwise the compartment holding most single-metabolite
reactions).
"""

from __future__ import annotations

import xml.etree.ElementTree as ET
from collections import Counter
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
from scipy.sparse import csr_matrix

DEFAULT_BOUND = 1000.0
_EXTERNAL_IDS = ("e", "C_e", "extracellular", "Extracellular", "ext")


def _local(tag):
    return tag.rsplit("}", 1)[-1]


def _attr(el, name):
    """Attribute by local name, whatever its namespace."""
    for key, value in el.attrib.items():
        if _local(key) == name:
            return value
    return None


def _number(text):
    t = str(text).strip()
    if t.upper() in ("INF", "+INF", "INFINITY"):
        return float("inf")
    if t.upper() in ("-INF", "-INFINITY"):
        return float("-inf")
    return float(t)


def _strip(prefix, value):
    return value[len(prefix):] if value.startswith(prefix) else value


@dataclass
class GenomeScaleModel:
    """One flux-balance model: ``S v = 0, lower <= v <= upper``, objective
    ``direction objective.v``."""

    id: str
    name: str
    metabolites: list
    compartments: list            # compartment of every metabolite
    reactions: list
    reaction_names: list
    S: csr_matrix
    lower: np.ndarray
    upper: np.ndarray
    objective: np.ndarray
    direction: str
    external_compartment: str | None
    exchanges: np.ndarray = field(default_factory=lambda: np.empty(0, np.int64))

    def reaction_index(self, rid):
        try:
            return self.reactions.index(rid)
        except ValueError:
            raise KeyError(rid) from None

    def metabolite_index(self, mid):
        try:
            return self.metabolites.index(mid)
        except ValueError:
            raise KeyError(mid) from None

    def reaction_stoichiometry(self, rid):
        col = self.S.tocsc()[:, self.reaction_index(rid)]
        return {self.metabolites[r]: float(v) for r, v in zip(col.indices, col.data)}

    def exchange_metabolite(self, col):
        """The single metabolite of exchange column ``col``."""
        rows = self.S.tocsc()[:, col].indices
        return self.metabolites[int(rows[0])]

    def fba_cost(self):
        """Minimisation cost of the FBA LP (``-c`` for a maximised
        objective, as ``src/dfba_simulator.py:1080`` passes to linprog)."""
        return -self.objective if self.direction == "max" else self.objective.copy()


def read_sbml(path) -> GenomeScaleModel:
    root = ET.parse(str(path)).getroot()
    model = next((el for el in root if _local(el.tag) == "model"), None)
    if model is None:
        raise ValueError(f"{path}: no <model> element")

    def section(name):
        for el in model:
            if _local(el.tag) == name:
                return list(el)
        return []

    comp_names = {c.get("id"): (c.get("name") or "") for c in section("listOfCompartments")}
    params = {}
    for p in section("listOfParameters"):
        if p.get("value") is not None:
            params[p.get("id")] = _number(p.get("value"))
    metabolites, compartments, row_of, boundary = [], [], {}, set()
    for sp in section("listOfSpecies"):
        sid = sp.get("id")
        if (sp.get("boundaryCondition") or "false").lower() == "true":
            boundary.add(sid)
            continue
        row_of[sid] = len(metabolites)
        metabolites.append(_strip("M_", sid))
        compartments.append(sp.get("compartment"))
    # FBC v1 flux bounds
    v1_bounds: dict[str, dict[str, float]] = {}
    for fb in section("listOfFluxBounds"):
        rid, op, val = _attr(fb, "reaction"), _attr(fb, "operation"), _number(_attr(fb, "value"))
        d = v1_bounds.setdefault(rid, {})
        if op in ("greaterEqual", "equal"):
            d["lower"] = val
        if op in ("lessEqual", "equal"):
            d["upper"] = val
    reactions, names, lower, upper = [], [], [], []
    rows, cols, vals = [], [], []
    sid_of_reaction = []
    for j, rx in enumerate(section("listOfReactions")):
        rid = rx.get("id")
        sid_of_reaction.append(rid)
        reactions.append(_strip("R_", rid))
        names.append(rx.get("name") or "")
        reversible = (rx.get("reversible") or "true").lower() == "true"
        acc: dict[int, float] = {}
        for part in rx:
            kind = _local(part.tag)
            if kind not in ("listOfReactants", "listOfProducts"):
                continue
            sign = -1.0 if kind == "listOfReactants" else 1.0
            for ref in part:
                s = ref.get("species")
                if s in boundary:
                    continue
                if s not in row_of:
                    raise ValueError(f"{path}: reaction {rid} uses unknown species {s}")
                st = float(ref.get("stoichiometry", "1"))
                acc[row_of[s]] = acc.get(row_of[s], 0.0) + sign * st
        for r, v in acc.items():
            if v != 0.0:
                rows.append(r)
                cols.append(j)
                vals.append(v)
        lo_ref, up_ref = _attr(rx, "lowerFluxBound"), _attr(rx, "upperFluxBound")
        for ref in (lo_ref, up_ref):
            if ref and ref not in params:
                raise ValueError(f"{path}: reaction {rid} references undefined bound parameter {ref}")
        lo = params[lo_ref] if lo_ref else v1_bounds.get(rid, {}).get("lower")
        up = params[up_ref] if up_ref else v1_bounds.get(rid, {}).get("upper")
        lo = (-DEFAULT_BOUND if reversible else 0.0) if lo is None else lo
        up = DEFAULT_BOUND if up is None else up
        if not lo <= up:
            raise ValueError(f"{path}: reaction {rid} has lower bound {lo} above upper bound {up}")
        lower.append(lo)
        upper.append(up)
    m, n = len(metabolites), len(reactions)
    S = csr_matrix((vals, (rows, cols)), shape=(m, n), dtype=np.float64)
    S.sum_duplicates()
    S.sort_indices()
    # active objective
    objective = np.zeros(n)
    direction = "max"
    col_of = {rid: j for j, rid in enumerate(sid_of_reaction)}
    objs = section("listOfObjectives")
    if objs:
        active = None
        for el in model:
            if _local(el.tag) == "listOfObjectives":
                active = _attr(el, "activeObjective")
        chosen = next((o for o in objs if _attr(o, "id") == active), objs[0])
        direction = "min" if (_attr(chosen, "type") or "maximize").startswith("min") else "max"
        for part in chosen:
            if _local(part.tag) != "listOfFluxObjectives":
                continue
            for fo in part:
                rid = _attr(fo, "reaction")
                if rid in col_of:
                    objective[col_of[rid]] += float(_attr(fo, "coefficient") or 1.0)
    # exchanges: single-metabolite reactions in the external compartment
    nnz_per_col = np.diff(S.tocsc().indptr)
    single = np.flatnonzero(nnz_per_col == 1)
    csc = S.tocsc()
    single_comp = [compartments[int(csc.indices[csc.indptr[j]])] for j in single]
    external = None
    present = set(compartments)
    for cid in _EXTERNAL_IDS:
        if cid in present:
            external = cid
            break
    if external is None:
        for cid in present:
            if "extracellular" in comp_names.get(cid, "").lower():
                external = cid
                break
    if external is None and single_comp:
        external = Counter(single_comp).most_common(1)[0][0]
    exchanges = np.array([j for j, c in zip(single, single_comp) if c == external], dtype=np.int64)
    return GenomeScaleModel(id=model.get("id") or Path(path).stem, name=model.get("name") or "",
                            metabolites=metabolites, compartments=compartments, reactions=reactions,
                            reaction_names=names, S=S, lower=np.asarray(lower, float), upper=np.asarray(upper, float),
                            objective=objective, direction=direction, external_compartment=external,
                            exchanges=exchanges)
