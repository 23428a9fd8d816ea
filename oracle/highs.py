"""HiGHS oracle (test infrastructure only).

The reference's exact CPU LP call is ``scipy.optimize.linprog(..., method=
"highs")`` on ``S v = 0`` (``src/dfba_simulator.py:1081-1091``); its batch
comparator maps ``linprog`` over a thread pool with one HiGHS thread per LP
(``scripts/microbatch_comparison_support.py:12-30``).  HiGHS version: the one
bundled with the installed SciPy (1.12.0 with SciPy 1.18.1); the reference
measured HiGHS 1.14.0 and pins ``highspy>=1.15.1`` -- optimal objective values
agree to LP tolerance regardless, only the vertex chosen on a degenerate face
can differ.
"""

from __future__ import annotations

import os
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np
from scipy.optimize import linprog


def solve_one(S, lower, upper, cost, rhs=None, neq=None, method="highs-ds"):
    """Solve ``min cost.x s.t. S[:neq] x = rhs[:neq], S[neq:] x <= rhs[neq:],
    lower <= x <= upper`` with HiGHS.  Returns ``(status, fun, x, y)`` with
    ``y`` the HiGHS row duals (equality rows then inequality rows)."""
    m = S.shape[0]
    rhs = np.zeros(m) if rhs is None else np.asarray(rhs, float)
    neq = m if neq is None else int(neq)
    kw = dict(bounds=np.column_stack([lower, upper]), method=method,
              options=dict(presolve=True))
    if neq:
        kw.update(A_eq=S[:neq], b_eq=rhs[:neq])
    if neq < m:
        kw.update(A_ub=S[neq:], b_ub=rhs[neq:])
    res = linprog(cost, **kw)
    if res.status != 0:
        return res.status, None, None, None
    y = []
    if neq:
        y.append(np.asarray(res.eqlin.marginals))
    if neq < m:
        y.append(np.asarray(res.ineqlin.marginals))
    y = np.concatenate(y) if y else np.empty(0)
    return 0, float(res.fun), np.asarray(res.x), y


def solve_batch(S_list, lowers, uppers, costs, *, workers=None, rhs_list=None, neq_list=None):
    """Solve a batch on ``workers`` threads, one HiGHS thread per LP.

    ``S_list`` etc. are per-instance sequences.  Returns a list of
    ``(status, fun, x, y)`` and the wall time.
    """
    workers = workers or len(os.sched_getaffinity(0))
    count = len(lowers)
    rhs_list = rhs_list or [None] * count
    neq_list = neq_list or [None] * count

    def one(i):
        return solve_one(S_list[i], lowers[i], uppers[i], costs[i], rhs_list[i], neq_list[i])

    start = time.perf_counter()
    with ThreadPoolExecutor(max_workers=workers) as pool:
        out = list(pool.map(one, range(count)))
    return out, time.perf_counter() - start
