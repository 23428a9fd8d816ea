"""Exact elimination of two-entry homogeneous equalities (presolve) and the
matching primal/dual postsolve.

Behaviour of the reference's ``HomogeneousEqualityReduction``
(``src/lp_equality_reduction.py:272-591``), restated: rows of the leading
equality block with exactly two nonzeros ``a x_p + b x_q = 0`` tie ``x_q`` to
``x_p``; rows that would close a cycle (union-find in row order), badly
scaled rows (coefficient ratio above ``max_scale_ratio``) and badly scaled
components stay as explicit equalities.  Every tree of the kept relations
becomes one reduced variable ``z_g`` with ``x_j = T_jg z_g`` (``T_jg`` the
tree's null-space weights normalised so its representative -- the largest
weight, lowest index -- has weight 1).  The reduced LP has matrix
``A[kept] T``, objective ``T^T c``, the intersected boxes of each tree's
columns and the kept rows.  The postsolve expands ``x = T z`` and lifts the
row duals: each reduced bound multiplier is charged to the original bound
that produced the tight endpoint (a "witness"), and the eliminated rows'
multipliers are solved from the trees' stationarity equations with a
precomputed sparse map.  Acceptance stays with the original LP's
certificate: nothing here solves or relaxes an LP.
"""

from __future__ import annotations

import hashlib

import numpy as np
from scipy.sparse import coo_matrix, csr_matrix, eye


def _canonical(problem):
    if not isinstance(problem, (tuple, list)) or len(problem) != 6:
        raise ValueError("Expected an (a, rhs, lower, upper, c, neq) LP tuple")
    a, rhs, lower, upper, c, neq = problem
    a = csr_matrix(a, dtype=np.float64, copy=True)
    a.sum_duplicates()
    a.eliminate_zeros()
    a.sort_indices()
    m, n = a.shape
    if n < 1 or not np.isfinite(a.data).all():
        raise ValueError("The LP matrix must have finite coefficients and columns")
    if isinstance(neq, (bool, np.bool_)) or not isinstance(neq, (int, np.integer)) or not 0 <= int(neq) <= m:
        raise ValueError("neq must identify an initial block of equality rows")
    out = []
    for name, v, size, finite in (("rhs", rhs, m, True), ("lower", lower, n, False), ("upper", upper, n, False),
                                  ("objective", c, n, True)):
        v = np.array(v, dtype=np.float64, copy=True)
        if v.shape != (size,):
            raise ValueError(f"{name} has the wrong shape")
        if np.isnan(v).any() or (finite and not np.isfinite(v).all()):
            raise ValueError(f"{name} contains invalid values")
        out.append(v)
    rhs, lower, upper, c = out
    if (lower > upper).any() or np.isposinf(lower).any() or np.isneginf(upper).any():
        raise ValueError("Invalid variable bounds")
    return a, rhs, lower, upper, c, int(neq)


def equality_fingerprint(a, neq) -> str:
    """Content hash of the equality block (shape, pattern, values, neq)."""
    e = csr_matrix(a[:neq])
    e.sum_duplicates()
    e.eliminate_zeros()
    e.sort_indices()
    h = hashlib.sha256()
    for name, value, dt in (("shape", e.shape, "<i8"), ("indptr", e.indptr, "<i8"), ("indices", e.indices, "<i8"),
                            ("data", e.data, "<f8"), ("neq", [neq], "<i8")):
        arr = np.asarray(value, dtype=dt)
        h.update(name.encode("ascii"))
        h.update(np.asarray(arr.shape, dtype="<i8").tobytes())
        h.update(arr.tobytes())
    return h.hexdigest()


class ReducedLP:
    """One LP reduced by a plan, with the witnesses its postsolve needs."""

    def __init__(self, plan, problem, original, kept_matrix, lower_witness, upper_witness):
        self.plan = plan
        self.problem = problem
        self.original_problem = original
        self.kept_matrix = kept_matrix
        self.lower_witness = lower_witness
        self.upper_witness = upper_witness
        self.fallback_witness = plan.representatives.copy()

    def expand_primal(self, z):
        return self.plan.expand_primal(z)

    def compress_primal(self, x, *, check=False, atol=1e-9):
        return self.plan.compress_primal(x, check=check, atol=atol)

    def allocate_bound_reduced_cost(self, reduced_cost):
        """Original-space bound multipliers: each reduced value sits on the
        witness of the reduced endpoint it belongs to (the representative
        when no finite original bound attains it)."""
        r = np.asarray(reduced_cost, dtype=np.float64)
        if r.shape != (self.plan.reduced_variables,) or not np.isfinite(r).all():
            raise ValueError("reduced_cost has the wrong shape or non-finite values")
        out = np.zeros(self.plan.original_variables)
        for g in np.flatnonzero(r != 0.0):
            w = int(self.lower_witness[g] if r[g] > 0.0 else self.upper_witness[g])
            if w < 0:
                w = int(self.fallback_witness[g])
            out[w] = r[g] / self.plan.weights[w]
        return out

    def lift_dual(self, reduced_y, reduced_cost):
        """Original row duals from the reduced row duals and reduced costs
        (``reduced_cost`` must be ``T^T (c - A[kept]^T reduced_y)``)."""
        plan = self.plan
        ry = np.asarray(reduced_y, dtype=np.float64)
        if ry.shape != (len(plan.kept_rows),) or not np.isfinite(ry).all():
            raise ValueError("reduced_y has the wrong shape or non-finite values")
        rc = np.asarray(reduced_cost, dtype=np.float64)
        if rc.shape != (plan.reduced_variables,) or not np.isfinite(rc).all():
            raise ValueError("reduced_cost has the wrong shape or non-finite values")
        a, _, _, _, c, _ = self.original_problem
        q = c - np.asarray(self.kept_matrix.T @ ry).ravel()
        expected = np.asarray(plan.transform.T @ q).ravel()
        if np.max(np.abs(expected - rc), initial=0.0) > 1e-10 * max(1.0, np.max(np.abs(expected), initial=0.0)):
            raise ValueError("reduced_cost is inconsistent with the reduced row dual")
        bound = self.allocate_bound_reduced_cost(rc)
        y = np.empty(a.shape[0])
        y[plan.kept_rows] = ry
        y[plan.eliminated_rows] = np.asarray(plan.dual_lift_map @ (q - bound)).ravel()
        if np.max(np.abs(c - np.asarray(a.T @ y).ravel() - bound), initial=0.0) > 1e-8:
            raise ArithmeticError("Eliminated equality dual lift lost original stationarity")
        return y


class EqualityReduction:
    """Fixed presolve plan of one equality block (see module docstring)."""

    def __init__(self, problem, *, max_scale_ratio=1e8):
        if isinstance(max_scale_ratio, (bool, np.bool_)) or not np.isfinite(max_scale_ratio) or \
                float(max_scale_ratio) < 1.0:
            raise ValueError("max_scale_ratio must be finite and at least one")
        a, rhs, lower, upper, c, neq = _canonical(problem)
        n = a.shape[1]
        self.original_shape = a.shape
        self.original_variables = n
        self.original_equalities = neq
        self.max_scale_ratio = float(max_scale_ratio)
        self.equality_fingerprint = equality_fingerprint(a, neq)

        # --- kept relations: two-entry homogeneous rows forming a forest ---
        root = np.arange(n)

        def find(v):
            while root[v] != v:
                root[v] = root[root[v]]
                v = root[v]
            return v

        edges = {}                       # row -> (p, q, a_p, a_q)
        touching = {}                    # node -> [(neighbour, row)]
        for r in range(neq):
            lo, hi = a.indptr[r], a.indptr[r + 1]
            if hi - lo != 2 or rhs[r] != 0.0:
                continue
            (p, q), (ap, aq) = a.indices[lo:hi], a.data[lo:hi]
            mags = np.abs([ap, aq])
            if mags.min() == 0.0 or mags.max() / mags.min() > self.max_scale_ratio:
                continue
            rp, rq = find(int(p)), find(int(q))
            if rp == rq:
                continue                 # closes a cycle: stays explicit
            root[max(rp, rq)] = min(rp, rq)
            edges[r] = (int(p), int(q), float(ap), float(aq))
            touching.setdefault(int(p), []).append((int(q), r))
            touching.setdefault(int(q), []).append((int(p), r))

        # --- trees and their null-space weights ---
        seen = set()
        trees = []
        for start in sorted(touching):
            if start in seen:
                continue
            alpha, members, rows, ok, stack = {start: 1.0}, [], set(), True, [start]
            while stack:
                v = stack.pop()
                if v in seen:
                    continue
                seen.add(v)
                members.append(v)
                for u, r in touching[v]:
                    rows.add(r)
                    if u in alpha:
                        continue
                    p, q, ap, aq = edges[r]
                    av, au = (ap, aq) if v == p else (aq, ap)
                    alpha[u] = -av * alpha[v] / au
                    if not np.isfinite(alpha[u]) or alpha[u] == 0.0:
                        ok = False
                    stack.append(u)
            mags = np.abs([alpha[v] for v in members])
            if not ok or len(members) < 2 or not np.isfinite(mags).all() or \
                    mags.max() / mags.min() > self.max_scale_ratio:
                continue
            top = mags.max()
            rep = min(v for v in members if abs(alpha[v]) == top)
            s = alpha[rep]
            weights = {v: alpha[v] / s for v in members}
            weights[rep] = 1.0
            trees.append((sorted(members), weights, sorted(rows), rep))
        in_tree = {v for t in trees for v in t[0]}
        groups = trees + [([v], {v: 1.0}, [], v) for v in range(n) if v not in in_tree]
        groups.sort(key=lambda t: t[0][0])

        # --- maps ---
        self.reduced_variables = len(groups)
        self.original_to_reduced = np.empty(n, dtype=np.int64)
        self.weights = np.empty(n)
        self.representatives = np.empty(len(groups), dtype=np.int64)
        tr, tc, tv, eliminated = [], [], [], []
        for g, (members, weights, rows, rep) in enumerate(groups):
            self.representatives[g] = rep
            eliminated += rows
            for v in members:
                self.original_to_reduced[v] = g
                self.weights[v] = weights[v]
                tr.append(v)
                tc.append(g)
                tv.append(weights[v])
        self.component_members = tuple(np.asarray(t[0], dtype=np.int64) for t in groups)
        self.transform = coo_matrix((tv, (tr, tc)), shape=(n, len(groups))).tocsr()
        self.T = self.transform
        norm2 = np.bincount(self.original_to_reduced, weights=self.weights ** 2, minlength=len(groups))
        self.compression = coo_matrix((self.weights / norm2[self.original_to_reduced],
                                       (self.original_to_reduced, np.arange(n))),
                                      shape=(len(groups), n)).tocsr()
        self.eliminated_rows = np.asarray(sorted(set(eliminated)), dtype=np.int64)
        gone = set(self.eliminated_rows.tolist())
        self.kept_rows = np.asarray([r for r in range(a.shape[0]) if r not in gone], dtype=np.int64)
        self.reduced_equalities = neq - len(self.eliminated_rows)
        self.dual_lift_map = self._tree_dual_map(edges, groups)
        # bound layout: per group, columns by decreasing |weight|, then index
        self._order = np.lexsort((np.arange(n), -np.abs(self.weights), self.original_to_reduced))
        self._starts = np.r_[0, np.flatnonzero(np.diff(self.original_to_reduced[self._order])) + 1]

        elim = a[self.eliminated_rows]
        if np.max(np.abs((elim @ self.transform).data), initial=0.0) > 1e-12:
            raise ArithmeticError("Constructed primal map is not in the equality null space")
        if len(self.eliminated_rows):
            err = self.dual_lift_map @ elim.T - eye(len(self.eliminated_rows), format="csr")
            if np.max(np.abs(err.data), initial=0.0) > 1e-10:
                raise ArithmeticError("Constructed tree dual map is not a left inverse of the eliminated transpose")

    from_problem = classmethod(lambda cls, problem, **kw: cls(problem, **kw))

    def _tree_dual_map(self, edges, groups):
        """Sparse map D with D A[eliminated]^T = I on the trees: the multiplier
        of the row joining a node to its parent (rooted at the
        representative) is that node's residual minus its children's rows'
        contributions, divided by the node's coefficient in that row."""
        pos = {r: i for i, r in enumerate(self.eliminated_rows)}
        expr = [None] * len(self.eliminated_rows)
        for members, _w, rows, rep in groups:
            if not rows:
                continue
            nbrs = {v: [] for v in members}
            for r in rows:
                p, q, _, _ = edges[r]
                nbrs[p].append((q, r))
                nbrs[q].append((p, r))
            parent_row = {rep: None}
            order = [rep]
            for v in order:
                for u, r in nbrs[v]:
                    if u not in parent_row:
                        parent_row[u] = r
                        order.append(u)
            if len(order) != len(members):
                raise ArithmeticError("Equality forest is disconnected")
            children = {v: [] for v in members}
            for v in order[1:]:
                p, q, _, _ = edges[parent_row[v]]
                children[q if v == p else p].append(v)
            for v in reversed(order[1:]):
                r = parent_row[v]
                p, q, ap, aq = edges[r]
                coef = ap if v == p else aq
                e = {v: 1.0 / coef}
                for ch in children[v]:
                    cr = parent_row[ch]
                    cp, cq, cap, caq = edges[cr]
                    f = -(cap if v == cp else caq) / coef
                    for k, val in expr[pos[cr]].items():
                        e[k] = e.get(k, 0.0) + f * val
                expr[pos[r]] = e
        rr, cc, vv = [], [], []
        for i, e in enumerate(expr):
            if e is None:
                raise ArithmeticError("Missing eliminated-row dual expression")
            for k in sorted(e):
                if e[k] != 0.0:
                    rr.append(i)
                    cc.append(k)
                    vv.append(e[k])
        return coo_matrix((vv, (rr, cc)), shape=(len(self.eliminated_rows), self.original_variables)).tocsr()

    def reduce(self, problem) -> ReducedLP:
        original = _canonical(problem)
        a, rhs, lower, upper, c, neq = original
        if a.shape != self.original_shape or neq != self.original_equalities:
            raise ValueError("LP dimensions/equality block changed from the reduction plan")
        if equality_fingerprint(a, neq) != self.equality_fingerprint:
            raise ValueError("Equality fingerprint changed from the reduction plan")
        if len(self.eliminated_rows) and np.any(rhs[self.eliminated_rows] != 0.0):
            raise ValueError("An eliminated equality is no longer homogeneous")
        w = self.weights
        pos = w > 0.0
        with np.errstate(over="raise", invalid="raise", divide="raise"):
            try:
                lo_ind = np.where(pos, lower, upper) / w
                up_ind = np.where(pos, upper, lower) / w
            except FloatingPointError as exc:
                raise ValueError("Reduced bound transformation overflowed or became invalid") from exc
        o, st = self._order, self._starts
        red_lo = np.maximum.reduceat(lo_ind[o], st)
        red_up = np.minimum.reduceat(up_ind[o], st)
        if np.any(red_lo > red_up):
            raise ValueError("Original bounds are infeasible under eliminated equalities")
        group_of = self.original_to_reduced[o]

        def witness(induced, endpoint):
            hit = np.isfinite(endpoint[group_of]) & (induced[o] == endpoint[group_of])
            first = np.minimum.reduceat(np.where(hit, np.arange(len(o)), len(o)), st)
            out = np.full(self.reduced_variables, -1, dtype=np.int64)
            found = first < len(o)
            out[found] = o[first[found]]
            return out

        kept = a[self.kept_rows].tocsr()
        red_a = (kept @ self.transform).tocsr()
        red_a.sum_duplicates()
        red_a.eliminate_zeros()
        red_a.sort_indices()
        reduced = (red_a, rhs[self.kept_rows].copy(), red_lo, red_up, np.asarray(self.transform.T @ c).ravel(),
                   self.reduced_equalities)
        return ReducedLP(self, reduced, original, kept, witness(lo_ind, red_lo), witness(up_ind, red_up))

    def compress_primal(self, x, *, check=False, atol=1e-9):
        """Least-squares reduced point of an original point (exact on the
        null space)."""
        x = np.asarray(x, dtype=np.float64)
        if x.shape[-1:] != (self.original_variables,) or not np.isfinite(x).all():
            raise ValueError("original_x has the wrong final dimension or non-finite values")
        z = np.asarray(self.compression @ x).ravel() if x.ndim == 1 else np.asarray(x @ self.compression.T)
        if check and not np.allclose(self.expand_primal(z), x, rtol=0.0, atol=atol):
            raise ValueError("original_x does not satisfy the eliminated equalities")
        return z

    def expand_primal(self, z):
        z = np.asarray(z, dtype=np.float64)
        if z.shape[-1:] != (self.reduced_variables,) or not np.isfinite(z).all():
            raise ValueError("reduced_x has the wrong final dimension or non-finite values")
        return np.asarray(self.transform @ z).ravel() if z.ndim == 1 else np.asarray(z @ self.transform.T)
