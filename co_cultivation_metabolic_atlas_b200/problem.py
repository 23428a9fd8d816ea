"""SciPy-``linprog`` request normalisation (host side of the boundary).

``normalize(c, kwargs)`` has the contract of the reference's ``_problem``
(``src/cpu_repeated_lp.py:119-147``) together with the checked path of
``split_variable_bounds`` (``src/lp_bounds.py:12-58``): it validates the
continuous ``linprog`` subset the simulator uses and returns
``(a, rhs, lower, upper, c, neq)`` with ``a = [A_eq; A_ub]`` as a canonical
CSR matrix (duplicates summed, zeros dropped, indices sorted).  Error
messages and the ``ValueError`` type follow the reference so callers see the
same failures.  ``request(problem)`` is the inverse used by traces
(``src/lp_trace.py:33-40``).
"""

from __future__ import annotations

import numpy as np
from scipy.sparse import csr_matrix, vstack


def split_bounds(bounds, variables):
    """Checked SciPy-style bounds: ``None`` -> ``[0, inf)``; one pair is
    broadcast; ``None`` inside a pair is an infinite bound."""
    if bounds is None:
        return np.zeros(variables), np.full(variables, np.inf)
    values = np.asarray(bounds)
    if values.shape == (2,):
        values = np.broadcast_to(values, (variables, 2))
    if values.shape != (variables, 2):
        raise ValueError('Bounds must be a pair or one pair per variable')
    if values.dtype.kind in 'biuf':
        return (np.array(values[:, 0], dtype=float, copy=True),
                np.array(values[:, 1], dtype=float, copy=True))
    values = np.asarray(bounds, dtype=object)
    if values.shape == (2,):
        values = np.broadcast_to(values, (variables, 2))
    lower = np.array([-np.inf if v is None else v for v in values[:, 0]], dtype=float)
    upper = np.array([np.inf if v is None else v for v in values[:, 1]], dtype=float)
    return lower, upper


def normalize(objective, kwargs):
    """Validate one ``(c, linprog kwargs)`` request; see module docstring."""
    c = np.asarray(objective, dtype=np.float64)
    if c.ndim != 1 or not len(c) or not np.isfinite(c).all():
        raise ValueError('A finite one-dimensional objective is required')
    n = len(c)
    integrality = kwargs.get('integrality')
    if integrality is not None and np.any(np.asarray(integrality)):
        raise ValueError('The batched engine supports continuous LPs only')
    if kwargs.get('method', 'highs-ds') not in ('highs', 'highs-ds'):
        raise ValueError('The request method must name HiGHS (highs or highs-ds)')
    blocks, rhs = [], []
    for matrix_name, rhs_name in (('A_eq', 'b_eq'), ('A_ub', 'b_ub')):
        supplied = kwargs.get(matrix_name)
        matrix = (csr_matrix((0, n), dtype=float) if supplied is None
                  else csr_matrix(supplied, dtype=float))
        if matrix.shape[1] != n or not np.isfinite(matrix.data).all():
            raise ValueError('Invalid LP matrix')
        values = kwargs.get(rhs_name)
        values = (np.empty(0) if values is None and not matrix.shape[0]
                  else np.asarray(values, dtype=float))
        if values.shape != (matrix.shape[0],) or not np.isfinite(values).all():
            raise ValueError('Each matrix row requires a finite RHS')
        blocks.append(matrix)
        rhs.append(values)
    a = vstack(blocks, format='csr')
    a.sum_duplicates()
    a.eliminate_zeros()
    a.sort_indices()
    neq = blocks[0].shape[0]
    lower, upper = split_bounds(kwargs.get('bounds'), n)
    if np.isnan(lower).any() or np.isnan(upper).any() or (lower > upper).any():
        raise ValueError('Invalid variable bounds')
    return a, np.concatenate(rhs), lower, upper, c.copy(), neq


def request(problem, *, stage=None):
    """``(a, rhs, lower, upper, c, neq)`` -> ``(c, linprog kwargs)``."""
    a, rhs, lower, upper, c, neq = problem
    kw = dict(A_eq=a[:neq], b_eq=rhs[:neq], A_ub=a[neq:], b_ub=rhs[neq:],
              bounds=np.column_stack((lower, upper)), method='highs-ds',
              options=dict(threads=1, parallel=False))
    if stage is not None:
        kw['_stage'] = stage
    return c, kw


def matrix_key(a, neq):
    """Content key of a canonical matrix (shape, pattern, values, neq)."""
    import hashlib
    h = hashlib.blake2b(digest_size=16)
    h.update(np.asarray(a.shape, dtype='<i8').tobytes())
    h.update(np.asarray([neq], dtype='<i8').tobytes())
    h.update(np.asarray(a.indptr, dtype='<i8').tobytes())
    h.update(np.asarray(a.indices, dtype='<i4').tobytes())
    h.update(np.asarray(a.data, dtype='<f8').tobytes())
    return h.hexdigest()
