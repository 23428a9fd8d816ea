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


def normalize(objective, kwargs, _cache=None):
    """Validate one ``(c, linprog kwargs)`` request; see module docstring.

    ``_cache`` (a dict owned by one ``normalize_batch`` call) maps the
    identities of the request's ``A_eq`` / ``A_ub`` objects to their
    canonical stacked matrix, and of its objective object to its validated
    copy, so requests that pass the same objects (every environment of a
    species in a dFBA rollout) canonicalise them once.
    """
    c_hit = None if _cache is None else _cache.get(('c', id(objective)))
    if c_hit is not None and c_hit[0] is objective:
        c = c_hit[1]
    else:
        c = np.asarray(objective, dtype=np.float64)
        if c.ndim != 1 or not len(c) or not np.isfinite(c).all():
            raise ValueError('A finite one-dimensional objective is required')
        c = c.copy()
        if _cache is not None:
            # the entry keeps the object alive, so its id stays its own
            _cache[('c', id(objective))] = (objective, c)
    n = len(c)
    integrality = kwargs.get('integrality')
    if integrality is not None and np.any(np.asarray(integrality)):
        raise ValueError('The batched engine supports continuous LPs only')
    if kwargs.get('method', 'highs-ds') not in ('highs', 'highs-ds'):
        raise ValueError('The request method must name HiGHS (highs or highs-ds)')
    supplied = (kwargs.get('A_eq'), kwargs.get('A_ub'))
    key = (id(supplied[0]), id(supplied[1]), n)
    hit = None if _cache is None else _cache.get(key)
    if hit is not None and not (hit[0][0] is supplied[0] and hit[0][1] is supplied[1]):
        hit = None
    blocks, rhs = [], []
    for k, rhs_name in enumerate(('b_eq', 'b_ub')):
        if hit is None:
            matrix = (csr_matrix((0, n), dtype=float) if supplied[k] is None
                      else csr_matrix(supplied[k], dtype=float))
            if matrix.shape[1] != n or not np.isfinite(matrix.data).all():
                raise ValueError('Invalid LP matrix')
            blocks.append(matrix)
            rows = matrix.shape[0]
        else:
            rows = hit[2][k]
        values = kwargs.get(rhs_name)
        values = (np.empty(0) if values is None and not rows
                  else np.asarray(values, dtype=float))
        if values.shape != (rows,) or not np.isfinite(values).all():
            raise ValueError('Each matrix row requires a finite RHS')
        rhs.append(values)
    if hit is None:
        a = vstack(blocks, format='csr')
        a.sum_duplicates()
        a.eliminate_zeros()
        a.sort_indices()
        shapes = (blocks[0].shape[0], blocks[1].shape[0])
        if _cache is not None:
            # the entry keeps the objects alive, so their ids stay theirs
            _cache[key] = (supplied, a, shapes)
    else:
        a, shapes = hit[1], hit[2]
    neq = shapes[0]
    lower, upper = split_bounds(kwargs.get('bounds'), n)
    if np.isnan(lower).any() or np.isnan(upper).any() or (lower > upper).any():
        raise ValueError('Invalid variable bounds')
    return a, np.concatenate(rhs), lower, upper, c, neq


def normalize_batch(requests):
    """``normalize`` of every request of one batch, canonicalising each
    distinct matrix and objective object once.  The returned problems of
    requests that share those objects share one canonical matrix and one
    objective copy (treat them as read-only)."""
    cache = {}
    return [normalize(c, kw, cache) for c, kw in requests]


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
