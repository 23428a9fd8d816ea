"""Original-LP certificate restated on the CPU (test infrastructure only).

Follows ``src/cpu_repeated_lp.py:150-178`` (``_certificate``) and the GPU
twin ``src/gpu_block_lp.py:52-132`` (``certify_blocks_device``):

* primal residual  = max(|A_eq x - b_eq|_inf, max(A_ub x - b_ub)+,
                         max(l - x)+, max(x - u)+)
* dual violation   = max(max(y_ub)+, reduced cost sign violations on infinite
                         bounds), reduced cost ``r = c - A^T y`` (HiGHS sign
                         convention, ``y_ub <= 0``)
* relative KKT gap = (sum |r (x - t)| + sum |y_ub (b - A x)_ub|) / max(1, |c.x|),
                     ``t = l`` where ``r >= 0`` else ``u`` (an infinite target
                     contributes zero)
* accepted iff primal <= 1e-5, dual <= 1e-7, gap <= 1e-7
  (``src/gpu_block_lp.py:84``).
"""

from __future__ import annotations

import numpy as np

PRIMAL_GATE = 1e-5
DUAL_GATE = 1e-7
GAP_GATE = 1e-7


def certificate(a, rhs, lower, upper, c, neq, x, y):
    x = np.asarray(x, dtype=float)
    y = np.asarray(y, dtype=float)
    if x.shape != c.shape or y.shape != rhs.shape or not np.isfinite(x).all() or not np.isfinite(y).all():
        return dict(primal_residual=np.inf, dual_violation=np.inf, relative_kkt_gap=np.inf,
                    objective=np.nan, certificate_passed=False)
    activity = a @ x
    reduced = c - a.T @ y
    row_error = activity - rhs
    primal = max(0.0, np.max(np.abs(row_error[:neq]), initial=0.0),
                 np.max(row_error[neq:], initial=0.0), np.max(lower - x, initial=0.0),
                 np.max(x - upper, initial=0.0))
    dual = max(0.0, np.max(y[neq:], initial=0.0),
               np.max(np.where(~np.isfinite(lower), reduced, 0.0), initial=0.0),
               np.max(np.where(~np.isfinite(upper), -reduced, 0.0), initial=0.0))
    target = np.where(reduced >= 0.0, lower, upper)
    bound_gap = np.abs(reduced * (x - np.where(np.isfinite(target), target, x))).sum()
    row_gap = np.abs(y[neq:] * (rhs - activity)[neq:]).sum()
    objective = float(c @ x)
    gap = (bound_gap + row_gap) / max(1.0, abs(objective))
    passed = bool(np.isfinite(gap) and primal <= PRIMAL_GATE and dual <= DUAL_GATE and gap <= GAP_GATE)
    return dict(primal_residual=float(primal), dual_violation=float(dual),
                relative_kkt_gap=float(gap), objective=objective, certificate_passed=passed,
                bound_complementarity_gap=float(bound_gap), row_complementarity_gap=float(row_gap))


def dual_objective(a, rhs, lower, upper, c, neq, y):
    """Lagrangian dual bound ``b.y + sum_j min over [l_j, u_j] of r_j x_j``
    with the reduced cost projected onto the directions the bounds allow
    (an infinite bound contributes zero and its sign violation is reported
    separately)."""
    r = c - a.T @ y
    term = np.where(r > 0, np.where(np.isfinite(lower), r * lower, 0.0),
                    np.where(r < 0, np.where(np.isfinite(upper), r * upper, 0.0), 0.0))
    return float(rhs @ y + term.sum())


def certificate_rows(a, rhs, lower, upper, c, neq, X, Y):
    """``certificate`` of many instances that share the matrix ``a``: row
    ``i`` of ``X`` / ``Y`` (and of ``rhs``, ``lower``, ``upper``, ``c`` when
    they are 2-D; 1-D ones are shared) is one instance.  Returns arrays of the
    primal residual, dual violation and relative KKT gap per instance, with
    the formulas (and operation order per instance) of ``certificate``."""
    X = np.asarray(X, dtype=float)
    Y = np.asarray(Y, dtype=float)
    E = X.shape[0]
    lower = np.broadcast_to(lower, X.shape)
    upper = np.broadcast_to(upper, X.shape)
    c = np.broadcast_to(c, X.shape)
    rhs = np.broadcast_to(rhs, Y.shape)
    activity = np.asarray((a @ X.T).T)
    reduced = c - np.asarray((a.T @ Y.T).T)
    row_error = activity - rhs
    zero = np.zeros(E)
    primal = np.maximum.reduce([zero,
                                np.abs(row_error[:, :neq]).max(axis=1, initial=0.0),
                                row_error[:, neq:].max(axis=1, initial=0.0),
                                (lower - X).max(axis=1, initial=0.0),
                                (X - upper).max(axis=1, initial=0.0)])
    dual = np.maximum.reduce([zero,
                              Y[:, neq:].max(axis=1, initial=0.0),
                              np.where(~np.isfinite(lower), reduced, 0.0).max(axis=1, initial=0.0),
                              np.where(~np.isfinite(upper), -reduced, 0.0).max(axis=1, initial=0.0)])
    target = np.where(reduced >= 0.0, lower, upper)
    bound_gap = np.abs(reduced * (X - np.where(np.isfinite(target), target, X))).sum(axis=1)
    row_gap = np.abs(Y[:, neq:] * (rhs - activity)[:, neq:]).sum(axis=1)
    objective = (c * X).sum(axis=1)
    gap = (bound_gap + row_gap) / np.maximum(1.0, np.abs(objective))
    return primal, dual, gap
