"""The reference's plain FP64 PDHG operator restated on the CPU (test
infrastructure only).

Metric (``src/gpu_pdhg_corrector.py:183-200``): ``sigma_i = eta / sum_j |A_ij|``
and ``tau_j = eta / sum_i |A_ij|`` (a zero row/column uses 1), then
``tau /= primal_weight`` and ``sigma *= primal_weight``.

Iteration (``src/gpu_pdhg_corrector.py:334-358``; the NumPy twin in the
reference's ``tests/test_gpu_pdhg_workspace.py:35-50``)::

    y  = min(y + sigma (b - A xbar), dual_upper)   dual_upper = 0 on ub rows
    x' = clip(x - tau (c - A^T y), l, u)
    xbar = x' + theta (x' - x);  x = x'
"""

from __future__ import annotations

import numpy as np
from scipy.sparse import csr_matrix


def metric(a, step_safety=0.99, primal_weight=1.0):
    a = csr_matrix(a, dtype=np.float64)
    absolute = abs(a)
    row_sum = np.asarray(absolute.sum(axis=1)).ravel()
    col_sum = np.asarray(absolute.sum(axis=0)).ravel()
    sigma = np.where(row_sum > 0.0, step_safety / np.where(row_sum > 0, row_sum, 1.0), 1.0)
    tau = np.where(col_sum > 0.0, step_safety / np.where(col_sum > 0, col_sum, 1.0), 1.0)
    return tau / primal_weight, sigma * primal_weight


def iterate(a, rhs, lower, upper, c, neq, iterations, *, x=None, y=None, step_safety=0.99,
            primal_weight=1.0, theta=1.0):
    a = csr_matrix(a, dtype=np.float64)
    m, n = a.shape
    tau, sigma = metric(a, step_safety, primal_weight)
    x = np.zeros(n) if x is None else np.asarray(x, float).copy()
    y = np.zeros(m) if y is None else np.asarray(y, float).copy()
    x = np.clip(x, lower, upper)
    dual_upper = np.where(np.arange(m) >= neq, 0.0, np.inf)
    y = np.minimum(y, dual_upper)
    xbar = x.copy()
    for _ in range(iterations):
        y = np.minimum(y + sigma * (rhs - a @ xbar), dual_upper)
        new_x = np.clip(x - tau * (c - a.T @ y), lower, upper)
        xbar = new_x + theta * (new_x - x)
        x = new_x
    return x, y
