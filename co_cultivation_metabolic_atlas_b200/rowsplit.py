"""Exact splitting of long matrix rows (presolve) and its postsolve.

Genome-scale models have a few hub metabolites (protons, water, ATP, ...)
whose balance rows hold hundreds to more than a thousand reactions, while
almost every other row holds fewer than ten.  The engine assigns one row per
lane of a 32-row slice, so a slice is as long as its longest row: one hub
row makes one warp walk a thousand entries per pass, and pads its slice to
32 times that length, which can push the whole matrix out of shared memory.

A row ``a.x (= or <=) b`` longer than ``max_length`` is split into ``k``
pieces: the first ``k - 1`` segments ``S_q`` of ``max_length`` entries get a
free variable each and an equality row ``a_{S_q}.x - z_q = 0``; the row
itself keeps its last segment plus ``sum_q z_q`` (same sense, same
right-hand side).  This is an exact reformulation:

* primal: ``x -> (x, z_q = a_{S_q}.x)``; restriction drops ``z``;
* dual: the segment rows take the row's dual (``y_seg = y_row`` is forced
  at optimality by the zero reduced cost of the free ``z``); restriction
  keeps the rows' duals, so reduced costs of ``x`` are the original ones
  wherever ``y_seg = y_row``.

Row order of the split LP: the original equality rows, then the segment
rows (equalities), then the original inequality rows; columns: the original
columns, then the segment variables.  Acceptance stays with the original
LP's certificate of the restricted pair.
"""

from __future__ import annotations

import numpy as np
from scipy.sparse import csr_matrix


class RowSplit:
    """Split plan of one matrix (and its equality count)."""

    def __init__(self, a, neq, max_length=64):
        a = csr_matrix(a, dtype=np.float64, copy=True)
        a.sum_duplicates()
        a.sort_indices()
        m, n = a.shape
        if not 0 <= int(neq) <= m:
            raise ValueError("neq must identify an initial block of equality rows")
        L = int(max_length)
        if L < 2:
            raise ValueError("max_length must be at least 2")
        self.m, self.n, self.neq0, self.max_length = m, n, int(neq), L
        lengths = np.diff(a.indptr)
        long_rows = np.flatnonzero(lengths > L)
        seg_row_of, seg_start, seg_stop = [], [], []
        for r in long_rows:
            k = -(-int(lengths[r]) // L)          # pieces: k - 1 segments + the kept tail
            for q in range(k - 1):
                seg_row_of.append(int(r))
                seg_start.append(int(a.indptr[r]) + q * L)
                seg_stop.append(int(a.indptr[r]) + (q + 1) * L)
        self.n_aux = len(seg_row_of)
        self.seg_row_of = np.asarray(seg_row_of, dtype=np.int64)
        S = self.n_aux
        # new row index of every original row
        self.row_map = np.where(np.arange(m) < self.neq0, np.arange(m), np.arange(m) + S).astype(np.int64)
        self.seg_rows = self.neq0 + np.arange(S, dtype=np.int64)
        self.neq = self.neq0 + S
        # assemble the split matrix
        kept = np.ones(a.nnz, dtype=bool)
        rows, cols, vals = [], [], []
        for q, (r, s0, s1) in enumerate(zip(seg_row_of, seg_start, seg_stop)):
            kept[s0:s1] = False
            rows.append(np.full(s1 - s0, self.seg_rows[q]))
            cols.append(a.indices[s0:s1])
            vals.append(a.data[s0:s1])
            rows.append([self.seg_rows[q]])                    # a_S.x - z_q = 0
            cols.append([n + q])
            vals.append([-1.0])
            rows.append([self.row_map[r]])                     # ... + z_q in the row itself
            cols.append([n + q])
            vals.append([1.0])
        coo_r = np.repeat(np.arange(m), lengths)
        rows.append(self.row_map[coo_r[kept]])
        cols.append(a.indices[kept])
        vals.append(a.data[kept])
        A = csr_matrix((np.concatenate(vals), (np.concatenate(rows).astype(np.int64), np.concatenate(cols))),
                       shape=(m + S, n + S))
        A.sum_duplicates()
        A.sort_indices()
        self.a = A
        self._seg = csr_matrix((a.data[~kept], (np.repeat(np.arange(S), L) if S else np.empty(0, np.int64),
                                                a.indices[~kept])), shape=(S, n)) if S else csr_matrix((0, n))

    @property
    def active(self):
        return self.n_aux > 0

    def split_problem(self, problem):
        """The split LP of ``(a, rhs, lower, upper, c, neq)`` (same matrix as
        the plan's)."""
        a, rhs, lower, upper, c, neq = problem
        if a.shape != (self.m, self.n) or int(neq) != self.neq0:
            raise ValueError("problem does not match the split plan")
        return (self.a, self.extend_rows(rhs, 0.0), self.extend_columns(lower, -np.inf),
                self.extend_columns(upper, np.inf), self.extend_columns(c, 0.0), self.neq)

    def extend_columns(self, v, fill):
        v = np.asarray(v, dtype=np.float64)
        return np.concatenate([v, np.full(v.shape[:-1] + (self.n_aux,), fill)], axis=-1)

    def extend_rows(self, v, fill):
        v = np.asarray(v, dtype=np.float64)
        out = np.full(v.shape[:-1] + (self.m + self.n_aux,), fill)
        out[..., self.row_map] = v
        return out

    def extend_primal(self, x):
        """``(x, z)`` with ``z_q`` the segment activities of ``x``."""
        x = np.asarray(x, dtype=np.float64)
        z = (self._seg @ x.T).T if self.n_aux else np.zeros(x.shape[:-1] + (0,))
        return np.concatenate([x, z], axis=-1)

    def extend_dual(self, y):
        """Row duals of the split LP: every segment row takes its row's dual."""
        y = np.asarray(y, dtype=np.float64)
        out = self.extend_rows(y, 0.0)
        out[..., self.seg_rows] = y[..., self.seg_row_of]
        return out

    def restrict(self, x, y):
        """Original-LP primal and row duals of a split-LP pair."""
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        return x[..., :self.n], y[..., self.row_map]
